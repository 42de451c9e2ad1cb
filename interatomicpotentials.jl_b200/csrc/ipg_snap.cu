// ipg_snap.cu — SNAP bispectrum pipeline on sm_100a (FP64).
//
// One thread block owns one centre atom at a time (persistent grid-stride loop) and
// keeps everything of that atom in shared memory:
//   phase 1  Utot = wself*I + sum_j sfac*w_j*U(r_ij)      (compute_ui.jl:5-175)
//            warps take neighbors, lanes take the entries of one level of the Wigner
//            recursion; per-warp partial sums are reduced across warps in fixed order.
//   phase 2  Z = CG (Utot x Utot) CG                       (compute_z.jl:1-62)
//            threads take Z entries; Utot is read from shared memory.
//   phase 3  B, E_i = beta[s_i] . B_i                       (compute_b.jl:67-157)
//   phase 4  Y = d(beta.B)/dU  (adjoint mode only)          (design of compute_yi.jl)
//   phase 5  per neighbor: U and dU/dr recomputed level by level, then
//            adjoint: dE_i/dr_ij = 2 sum Re(conj(dU) Y)    (design of compute_dij.jl)
//            plain:   dB_i/dr_ij, 3 CG-symmetry terms       (compute_b.jl:166-404),
//                     written out per directed pair (the materialised dB/dr)
//            vjp:     V_i = sum_j (g_i - g_j) . dU_ij, then dB-contraction with Z.
// The per-pair results are scattered to atoms by a gather over the CSR list and its
// transpose, so every reduction is in a fixed order (bitwise reproducible).
#include <algorithm>

#include <cstdio>
#include <cstdlib>
#include <string>

#include "ipg_snap.cuh"
#include "ipg_snap_chain.cuh"

namespace {

// MODE_ADJY: the adjoint per-atom part alone (Z, weighted Y out, E from Y); the
// per-neighbor part runs in k_snap_pair_adj.  MODE_ADJ: the whole adjoint in one block
// (twojmax beyond the register-chain kernels).
enum SnapMode { MODE_DESC = 0, MODE_ADJ = 1, MODE_PLAIN = 2, MODE_VJP = 3, MODE_ADJY = 4 };

inline unsigned nblk(int64_t n, int t) { return (unsigned)std::max<int64_t>(1, (n + t - 1) / t); }

struct SnapIO {
  int64_t n;
  const int64_t* off;       // [n+1] neighbor CSR
  const int32_t* nbr;       // [np]
  const double* rij;        // [np][3]  x_j - x_i
  const int32_t* species;   // [n]
  double* Ei;               // [n] beta[s_i].B_i (without beta0)
  double* B;                // [n][K] or null
  double* fvec;             // [np][3]  adjoint dE_i/dr_ij
  double* dbl;              // [np][K][3] plain dB_i/dr_ij
  const double* g;          // [n][3] VJP cotangent of forces
  double gE;                // VJP cotangent of energy
  double* gpart;            // [gridDim][nsp*K] VJP partials
  double2* yout;            // [n][u_half] adjoint: weighted Y written out for the pair kernel
  const double2* utot_in;   // [n][idxu_max] Utot from k_snap_utot (phase 1 skipped) or null
  int* status;
};

// Whether the per-atom kernel needs the per-warp level buffers (its own phase 1 or the
// in-block per-neighbor phase 5).
__host__ __device__ inline bool needs_levels(int mode, bool has_utot, bool has_yout) {
  return !(has_utot && (mode == MODE_DESC || mode == MODE_ADJY || (mode == MODE_ADJ && has_yout)));
}

// Species ids are validated by the neighbor build (status word); clamping here keeps a
// bad id from indexing the per-species tables.
__device__ __forceinline__ int clamp_sp(int s, int nsp) { return s < 0 ? 0 : (s >= nsp ? nsp - 1 : s); }

__device__ __forceinline__ double2 cmul_conj(double2 a, double2 v) {  // conj(a) * v
  return make_double2(a.x * v.x + a.y * v.y, a.x * v.y - a.y * v.x);
}

__device__ __forceinline__ double sfac_of(const SnapDev& S, double r, double rcut) {  // compute_ui.jl:350-364
  if (!S.switch_flag) return 1.0;
  if (r <= S.rmin0) return 1.0;
  if (r > rcut) return 0.0;
  return 0.5 * (cos((r - S.rmin0) * (M_PI / (rcut - S.rmin0))) + 1.0);
}
__device__ __forceinline__ double dsfac_of(const SnapDev& S, double r, double rcut) {  // compute_ui.jl:366-380
  if (!S.switch_flag) return 0.0;
  if (r <= S.rmin0) return 0.0;
  double rcutfac = M_PI / (rcut - S.rmin0);
  return -0.5 * (sin((r - S.rmin0) * rcutfac) * rcutfac);
}

// Number of weight-1 half-plane entries of level l (rows 2mb < l, plus ma < l/2 of the
// middle row for even l); the middle element of an even level has weight 1/2.
__device__ __forceinline__ int nfull_of(int l) { return ((l + 1) / 2) * (l + 1) + ((l & 1) ? 0 : l / 2); }

// Per-pair geometry for the derivative recursion (compute_duidrj, compute_ui.jl:328-347
// and the prologue of compute_duarray, :191-216).
struct PairGeom {
  double2 a, b;
  double2 da[3], db[3];
  double u[3];
  double sfac, dsfac;
};

__device__ __forceinline__ void geom_du(const SnapDev& S, double x, double y, double z, double rcut, double wj,
                                        PairGeom& G) {
  double rsq = x * x + y * y + z * z;
  double r = sqrt(rsq);
  double rscale0 = S.rfac0 * M_PI / (rcut - S.rmin0);
  double theta0 = (r - S.rmin0) * rscale0;
  double sn, cs;
  sincos(theta0, &sn, &cs);
  double z0 = r * cs / sn;
  double dz0dr = z0 / r - (r * rscale0) * (rsq + z0 * z0) / rsq;
  double rinv = 1.0 / r;
  G.u[0] = x * rinv;
  G.u[1] = y * rinv;
  G.u[2] = z * rinv;
  double r0inv = 1.0 / sqrt(r * r + z0 * z0);
  G.a = make_double2(z0 * r0inv, -z * r0inv);
  G.b = make_double2(y * r0inv, -x * r0inv);
  double dr0invdr = -r0inv * r0inv * r0inv * (r + z0 * dz0dr);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    double dr0 = dr0invdr * G.u[k];
    double dz0 = dz0dr * G.u[k];
    G.da[k] = make_double2(dz0 * r0inv + z0 * dr0, -z * dr0);
    G.db[k] = make_double2(y * dr0, -x * dr0);
  }
  G.da[2].y += -r0inv;
  G.db[0].y += -r0inv;
  G.db[1].x += r0inv;
  G.sfac = sfac_of(S, r, rcut) * wj;
  G.dsfac = dsfac_of(S, r, rcut) * wj;
}

// One level of the Wigner recursion (compute_ui.jl:66-101, derivative :224-267) for
// `ncomp` components (1: U only; 4: U and dU/dx, dU/dy, dU/dz), lanes over
// (component, entry).  prev holds level j-1 rows 0..j/2 (row length j), cur receives
// level j rows 0..j/2 (row length j+1) and, for odd j, the mirrored row (j+1)/2
// (inversion symmetry, compute_ui.jl:105-125).  Buffers are [comp][ext_max].
__device__ __forceinline__ void wigner_level(const SnapDev& S, const double* rpq, int j, int ncomp,
                                             const PairGeom& G, const double2* __restrict__ prev,
                                             double2* __restrict__ cur, int lane) {
  const int J2 = S.J + 2;
  const int em = S.ext_max;
  const int nrec = (j / 2 + 1) * (j + 1);
  for (int t = lane; t < ncomp * nrec; t += 32) {
    int comp = t / nrec;
    int e = t - comp * nrec;
    int mb = e / (j + 1);
    int ma = e - mb * (j + 1);
    double2 dA = make_double2(0.0, 0.0), dB = make_double2(0.0, 0.0);
    if (comp == 1) { dA = G.da[0]; dB = G.db[0]; }
    if (comp == 2) { dA = G.da[1]; dB = G.db[1]; }
    if (comp == 3) { dA = G.da[2]; dB = G.db[2]; }
    double2 res = make_double2(0.0, 0.0);
    if (ma > 0) {  // -rootpq[ma][j-mb] * conj(b) * u_{j-1}[mb][ma-1]
      double rp = rpq[ma * J2 + (j - mb)];
      double2 v = prev[mb * j + ma - 1];
      double2 t1 = cmul_conj(G.b, v);
      if (comp) {
        double2 dv = prev[comp * em + mb * j + ma - 1];
        double2 t2 = cmul_conj(dB, v);
        double2 t3 = cmul_conj(G.b, dv);
        t1 = make_double2(t2.x + t3.x, t2.y + t3.y);
      }
      res = make_double2(-rp * t1.x, -rp * t1.y);
    }
    if (ma < j) {  // + rootpq[j-ma][j-mb] * conj(a) * u_{j-1}[mb][ma]
      double rp = rpq[(j - ma) * J2 + (j - mb)];
      double2 v = prev[mb * j + ma];
      double2 t1 = cmul_conj(G.a, v);
      if (comp) {
        double2 dv = prev[comp * em + mb * j + ma];
        double2 t2 = cmul_conj(dA, v);
        double2 t3 = cmul_conj(G.a, dv);
        t1 = make_double2(t2.x + t3.x, t2.y + t3.y);
      }
      res.x += rp * t1.x;
      res.y += rp * t1.y;
    }
    cur[comp * em + e] = res;
  }
  __syncwarp();
  if (j & 1) {  // u[R][c] = (-1)^(c+R) conj(u[j-R][j-c]),  R = (j+1)/2
    const int R = (j + 1) / 2;
    for (int t = lane; t < ncomp * (j + 1); t += 32) {
      int comp = t / (j + 1);
      int c = t - comp * (j + 1);
      double2 src = cur[comp * em + (j - R) * (j + 1) + (j - c)];
      double sg = ((c + R) & 1) ? -1.0 : 1.0;
      cur[comp * em + R * (j + 1) + c] = make_double2(sg * src.x, -sg * src.y);
    }
    __syncwarp();
  }
}

// Shared-memory layout (doubles, 16-byte aligned blocks).
struct SmemLayout {
  size_t ut, zs, ys, bs, rpq, lv, duf, gacc, total;
};

__host__ __device__ inline size_t al16(size_t x) { return (x + 1) & ~size_t(1); }  // in doubles

__host__ __device__ inline SmemLayout smem_layout(const SnapDev& S, int nwarps, int mode, bool levels) {
  SmemLayout L;
  size_t o = 0;
  L.ut = o;
  o += al16(2 * (size_t)S.idxu_max);
  L.zs = o;  // Z; phase 1 reuses it for the per-warp partial sums of Utot
  const size_t zsz = 2 * (size_t)S.idxz_max, usz = 2 * (size_t)nwarps * S.u_half;
  o += al16(zsz > usz ? zsz : usz);
  L.ys = o;  // Y (adjoint) or V (vjp)
  o += al16(2 * (size_t)S.u_half);
  L.bs = o;
  o += al16((size_t)S.K);
  L.rpq = o;
  o += al16((size_t)(S.J + 2) * (S.J + 2));
  L.lv = o;  // per warp: 2 levels x 4 components x ext_max complex
  if (levels) o += al16((size_t)nwarps * 2 * 4 * 2 * S.ext_max);
  L.duf = o;  // plain: per-warp dU/dr [3][u_half]; vjp: per-warp partial V [u_half]
  if (mode == MODE_PLAIN) o += al16((size_t)nwarps * 2 * 3 * S.u_half);
  if (mode == MODE_VJP) o += al16((size_t)nwarps * 2 * S.u_half);
  L.gacc = o;
  if (mode == MODE_VJP) o += al16((size_t)S.nsp * S.K);
  L.total = o * sizeof(double);
  return L;
}

template <int MODE>
__global__ void __launch_bounds__(256) k_snap_atom(const __grid_constant__ SnapDev S, SnapIO io) {
  extern __shared__ double smem[];
  const int nwarps = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const SmemLayout L = smem_layout(S, nwarps, MODE, needs_levels(MODE, io.utot_in != nullptr, io.yout != nullptr));
  double2* ut = reinterpret_cast<double2*>(smem + L.ut);
  double2* zs = reinterpret_cast<double2*>(smem + L.zs);
  double2* ys = reinterpret_cast<double2*>(smem + L.ys);
  double* bs = smem + L.bs;
  double* rpq = smem + L.rpq;
  double2* lvw = reinterpret_cast<double2*>(smem + L.lv) + (size_t)warp * 2 * 4 * S.ext_max;
  double2* lv0 = lvw;
  double2* lv1 = lvw + 4 * S.ext_max;
  double* gacc = smem + L.gacc;
  const int J = S.J, K = S.K, uh = S.u_half;

  for (int q = threadIdx.x; q < (J + 2) * (J + 2); q += blockDim.x) rpq[q] = S.rootpq[q];
  if (MODE == MODE_VJP)
    for (int q = threadIdx.x; q < S.nsp * K; q += blockDim.x) gacc[q] = 0.0;
  __syncthreads();

  for (int64_t i = blockIdx.x; i < io.n; i += gridDim.x) {
    const int64_t beg = io.off[i], end = io.off[i + 1];
    const int si = clamp_sp(io.species[i], S.nsp);

    // ---------------- phase 1: Utot (half plane) ----------------
    if (io.utot_in) {  // computed by k_snap_utot
      const double2* src = io.utot_in + (size_t)i * S.idxu_max;
      for (int q = threadIdx.x; q < S.idxu_max; q += blockDim.x) ut[q] = src[q];
      __syncthreads();
    } else {
    double2* upart = zs;  // [nwarps][u_half]
    for (int q = threadIdx.x; q < nwarps * uh; q += blockDim.x) upart[q] = make_double2(0.0, 0.0);
    __syncthreads();
    {
      double2* up = upart + (size_t)warp * uh;
      for (int64_t p = beg + warp; p < end; p += nwarps) {
        const double x = io.rij[3 * p], y = io.rij[3 * p + 1], z = io.rij[3 * p + 2];
        const int sj = clamp_sp(io.species[io.nbr[p]], S.nsp);
        const double rcut = (S.radii[si] + S.radii[sj]) * S.rcutfac;  // runtime_arrays.jl:50
        const double rsq = x * x + y * y + z * z;
        const double r = sqrt(rsq);
        const double theta0 = (r - S.rmin0) * S.rfac0 * M_PI / (rcut - S.rmin0);
        const double z0 = r / tan(theta0);
        const double r0inv = 1.0 / sqrt(r * r + z0 * z0);
        PairGeom G;
        G.a = make_double2(r0inv * z0, -r0inv * z);
        G.b = make_double2(r0inv * y, -r0inv * x);
        const double sw = sfac_of(S, r, rcut) * S.weight[sj];
        double2* prev = lv0;
        double2* cur = lv1;
        if (lane == 0) {
          prev[0] = make_double2(1.0, 0.0);
          up[0].x += sw;
        }
        __syncwarp();
        for (int j = 1; j <= J; j++) {
          wigner_level(S, rpq, j, 1, G, prev, cur, lane);
          const int nrec = (j / 2 + 1) * (j + 1);
          double2* upj = up + S.half_block[j];
          for (int e = lane; e < nrec; e += 32) {
            double2 v = cur[e];
            upj[e].x += sw * v.x;
            upj[e].y += sw * v.y;
          }
          __syncwarp();
          double2* t = prev;
          prev = cur;
          cur = t;
        }
      }
    }
    __syncthreads();
    // cross-warp sum (fixed order) + wself diagonal + inversion-symmetric fill
    for (int h = threadIdx.x; h < uh; h += blockDim.x) {
      double2 s = make_double2(0.0, 0.0);
      for (int w = 0; w < nwarps; w++) {
        double2 v = upart[(size_t)w * uh + h];
        s.x += v.x;
        s.y += v.y;
      }
      int j = 0;
      while (j < J && S.half_block[j + 1] <= h) j++;
      int e = h - S.half_block[j];
      int mb = e / (j + 1), ma = e - mb * (j + 1);
      if (ma == mb) s.x += S.wself;
      const int ub = S.idxu_block[j];
      const bool middle = (2 * mb == j);
      if (middle && ma > mb) continue;  // written as the mirror of ma' = j - ma
      ut[ub + mb * (j + 1) + ma] = s;
      if (!(middle && ma == mb)) {
        double sg = ((ma + mb) & 1) ? -1.0 : 1.0;
        ut[ub + (j - mb) * (j + 1) + (j - ma)] = make_double2(sg * s.x, -sg * s.y);
      }
    }
    __syncthreads();
    }  // phase 1

    // ---------------- phase 2: Z ----------------
    for (int t = threadIdx.x; t < S.idxz_max; t += blockDim.x) {
      const int jjz = S.zperm[t];
      const ZDev q = S.idxz[jjz];
      const double* cgb = S.cglist + q.cgoff;
      const int j1 = q.j1, j2 = q.j2;
      double zr = 0.0, zi = 0.0;
      int i1 = q.u1base, i2 = q.u2base, icgb = q.icgb0;
      for (int ib = 0; ib < q.nb; ib++) {
        double sr = 0.0, sim = 0.0;
        int icga = q.icga0;
        for (int ia = 0; ia < q.na; ia++) {
          const double2 u1 = ut[i1 + ia];
          const double2 u2 = ut[i2 - ia];
          const double c = __ldg(cgb + icga);
          sr += c * (u1.x * u2.x - u1.y * u2.y);
          sim += c * (u1.x * u2.y + u1.y * u2.x);
          icga += j2;
        }
        const double cb = __ldg(cgb + icgb);
        zr += cb * sr;
        zi += cb * sim;
        i1 += j1 + 1;
        i2 -= j2 + 1;
        icgb += j2;
      }
      if (S.bnorm_flag) {
        zr /= (q.j + 1);
        zi /= (q.j + 1);
      }
      zs[jjz] = make_double2(zr, zi);
    }
    __syncthreads();

    if (MODE == MODE_ADJY) {
      // Y' = w Y (half-plane weights folded in) out, and E_i from Y: B is cubic in U, so
      // beta.B = (2/3) sum_h w_h Re(conj(U_h) Y_h) (Euler's theorem), minus beta.bzero.
      __shared__ double red[32];
      const double* yc = S.ycoef + (size_t)si * S.idxz_max;
      double e = 0.0;
      for (int h = threadIdx.x; h < uh; h += blockDim.x) {
        int j = 0;
        while (j < J && S.half_block[j + 1] <= h) j++;
        const int ee = h - S.half_block[j], mb = ee / (j + 1), ma = ee - mb * (j + 1);
        const double w = (2 * mb < j) ? 1.0 : (ma < mb ? 1.0 : (ma == mb ? 0.5 : 0.0));
        double2 y = make_double2(0.0, 0.0);
        if (w != 0.0)
          for (int q = S.y_off[h]; q < S.y_off[h + 1]; q++) {
            const int jjz = S.y_jjz[q];
            const double c = yc[jjz];
            const double2 zz = zs[jjz];
            y.x += c * zz.x;
            y.y += c * zz.y;
          }
        y.x *= w;
        y.y *= w;
        io.yout[(size_t)h * io.n + i] = y;
        const double2 u = ut[S.idxu_block[j] + ee];
        e += u.x * y.x + u.y * y.y;
      }
      e = warp_sum(e);
      if (lane == 0) red[warp] = e;
      __syncthreads();
      if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < nwarps; w++) t += red[w];
        io.Ei[i] = (2.0 / 3.0) * t + S.ebias[si];
      }
      __syncthreads();
      continue;
    }

    // ---------------- phase 3: B and E_i ----------------
    for (int b = threadIdx.x; b < K; b += blockDim.x) {
      const DBDev d = S.db[b];
      const int l = d.l[0], z0 = d.z0[0], u0 = S.idxu_block[l];
      const int nf = nfull_of(l);
      double s = 0.0;
      for (int e = 0; e < nf; e++) {
        double2 u = ut[u0 + e], zz = zs[z0 + e];
        s += u.x * zz.x + u.y * zz.y;
      }
      if (!(l & 1)) {
        int e = (l / 2) * (l + 1) + l / 2;
        double2 u = ut[u0 + e], zz = zs[z0 + e];
        s += 0.5 * (u.x * zz.x + u.y * zz.y);
      }
      double Bv = 2.0 * s - (S.bzero_flag ? S.bzero[l] : 0.0);
      bs[b] = Bv;
      if (io.B) io.B[i * K + b] = Bv;
    }
    __syncthreads();
    if (warp == 0) {
      double e = 0.0;
      const double* bt = S.beta + (size_t)si * K;
      for (int b = lane; b < K; b += 32) e += bt[b] * bs[b];
      e = warp_sum(e);
      if (lane == 0) io.Ei[i] = e;
    }

    if (MODE == MODE_DESC) {
      __syncthreads();
      continue;
    }

    // ---------------- phase 4: Y (adjoint) / zero V (vjp) ----------------
    if (MODE == MODE_ADJ) {
      const double* yc = S.ycoef + (size_t)si * S.idxz_max;
      for (int h = threadIdx.x; h < uh; h += blockDim.x) {
        double2 s = make_double2(0.0, 0.0);
        for (int q = S.y_off[h]; q < S.y_off[h + 1]; q++) {
          int jjz = S.y_jjz[q];
          double c = yc[jjz];
          double2 zz = zs[jjz];
          s.x += c * zz.x;
          s.y += c * zz.y;
        }
        ys[h] = s;
      }
    }
    double2* vall = reinterpret_cast<double2*>(smem + L.duf);  // VJP: [nwarps][u_half]
    if (MODE == MODE_VJP)
      for (int q = threadIdx.x; q < nwarps * uh; q += blockDim.x) vall[q] = make_double2(0.0, 0.0);
    __syncthreads();

    // ---------------- phase 5: per-neighbor derivatives ----------------
    double2* dufw = reinterpret_cast<double2*>(smem + L.duf) + (size_t)warp * 3 * uh;  // [3][u_half]
    double2* vw = vall + (size_t)warp * uh;
    double gi[3] = {0.0, 0.0, 0.0};
    if (MODE == MODE_VJP) {
      gi[0] = io.g[3 * i];
      gi[1] = io.g[3 * i + 1];
      gi[2] = io.g[3 * i + 2];
    }
    for (int64_t p = beg + warp; p < end; p += nwarps) {
      const int32_t jn = io.nbr[p];
      const int sj = clamp_sp(io.species[jn], S.nsp);
      const double rcut = (S.radii[si] + S.radii[sj]) * S.rcutfac;
      PairGeom G;
      geom_du(S, io.rij[3 * p], io.rij[3 * p + 1], io.rij[3 * p + 2], rcut, S.weight[sj], G);
      double gv[3] = {0.0, 0.0, 0.0};
      if (MODE == MODE_VJP) {
        gv[0] = gi[0] - io.g[3 * jn];
        gv[1] = gi[1] - io.g[3 * jn + 1];
        gv[2] = gi[2] - io.g[3 * jn + 2];
      }
      double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
      double2* prev = lv0;
      double2* cur = lv1;
      const int em = S.ext_max;
      for (int j = 0; j <= J; j++) {
        if (j == 0) {
          if (lane < 4) cur[lane * em] = make_double2(lane == 0 ? 1.0 : 0.0, 0.0);
          __syncwarp();
        } else {
          wigner_level(S, rpq, j, 4, G, prev, cur, lane);
        }
        const int nrec = (j / 2 + 1) * (j + 1);
        const int hb = S.half_block[j];
        if (MODE == MODE_ADJ) {
          const int nf = nfull_of(j);
          const int emid = (j & 1) ? -1 : (j / 2) * (j + 1) + j / 2;
          for (int e = lane; e < nrec; e += 32) {
            double w = (e < nf) ? 1.0 : (e == emid ? 0.5 : 0.0);
            if (w == 0.0) continue;
            double2 u = cur[e];
            double2 Y = ys[hb + e];
            double2 d0 = cur[em + e], d1 = cur[2 * em + e], d2 = cur[3 * em + e];
            acc0 += w * ((G.dsfac * u.x * G.u[0] + G.sfac * d0.x) * Y.x + (G.dsfac * u.y * G.u[0] + G.sfac * d0.y) * Y.y);
            acc1 += w * ((G.dsfac * u.x * G.u[1] + G.sfac * d1.x) * Y.x + (G.dsfac * u.y * G.u[1] + G.sfac * d1.y) * Y.y);
            acc2 += w * ((G.dsfac * u.x * G.u[2] + G.sfac * d2.x) * Y.x + (G.dsfac * u.y * G.u[2] + G.sfac * d2.y) * Y.y);
          }
        } else if (MODE == MODE_PLAIN) {
          for (int e = lane; e < nrec; e += 32) {
            double2 u = cur[e];
#pragma unroll
            for (int k = 0; k < 3; k++) {
              double2 d = cur[(k + 1) * em + e];
              dufw[k * uh + hb + e] = make_double2(G.dsfac * u.x * G.u[k] + G.sfac * d.x,
                                                   G.dsfac * u.y * G.u[k] + G.sfac * d.y);
            }
          }
        } else if (MODE == MODE_VJP) {
          for (int e = lane; e < nrec; e += 32) {
            double2 u = cur[e];
            double vx = 0.0, vy = 0.0;
#pragma unroll
            for (int k = 0; k < 3; k++) {
              double2 d = cur[(k + 1) * em + e];
              vx += gv[k] * (G.dsfac * u.x * G.u[k] + G.sfac * d.x);
              vy += gv[k] * (G.dsfac * u.y * G.u[k] + G.sfac * d.y);
            }
            vw[hb + e].x += vx;  // this lane owns entry e of this warp's partial
            vw[hb + e].y += vy;
          }
        }
        __syncwarp();
        double2* t = prev;
        prev = cur;
        cur = t;
      }
      if (MODE == MODE_ADJ) {
        acc0 = warp_sum(acc0);
        acc1 = warp_sum(acc1);
        acc2 = warp_sum(acc2);
        if (lane == 0) {
          io.fvec[3 * p] = 2.0 * acc0;
          io.fvec[3 * p + 1] = 2.0 * acc1;
          io.fvec[3 * p + 2] = 2.0 * acc2;
        }
      } else if (MODE == MODE_PLAIN) {
        double* out = io.dbl + (size_t)p * K * 3;
        for (int t = lane; t < 3 * K; t += 32) {
          const int b = t / 3, k = t - 3 * b;
          const DBDev d = S.db[b];
          double tot = 0.0;
#pragma unroll
          for (int term = 0; term < 3; term++) {
            const int l = d.l[term], z0 = d.z0[term], hb = S.half_block[l];
            const int nf = nfull_of(l);
            const double2* du = dufw + k * uh + hb;
            double s = 0.0;
            for (int e = 0; e < nf; e++) {
              double2 a = du[e], zz = zs[z0 + e];
              s += a.x * zz.x + a.y * zz.y;
            }
            if (!(l & 1)) {
              int e = (l / 2) * (l + 1) + l / 2;
              double2 a = du[e], zz = zs[z0 + e];
              s += 0.5 * (a.x * zz.x + a.y * zz.y);
            }
            tot += d.fac[term] * s;
          }
          out[t] = 2.0 * tot;
        }
        __syncwarp();
      }
    }
    __syncthreads();

    if (MODE == MODE_VJP) {
      // V = sum of the per-warp partials (fixed order)
      double2* vpart = ys;
      for (int h = threadIdx.x; h < uh; h += blockDim.x) {
        double2 v = make_double2(0.0, 0.0);
        for (int w = 0; w < nwarps; w++) {
          v.x += vall[(size_t)w * uh + h].x;
          v.y += vall[(size_t)w * uh + h].y;
        }
        vpart[h] = v;
      }
      __syncthreads();
      // gbeta[s_i][b] += gE * B_i[b] + 2 sum_terms fac * sum_half Re(conj(V) Z)
      for (int b = threadIdx.x; b < K; b += blockDim.x) {
        const DBDev d = S.db[b];
        double tot = 0.0;
        for (int term = 0; term < 3; term++) {
          const int l = d.l[term], z0 = d.z0[term], hb = S.half_block[l];
          const int nf = nfull_of(l);
          double s = 0.0;
          for (int e = 0; e < nf; e++) {
            double2 a = vpart[hb + e], zz = zs[z0 + e];
            s += a.x * zz.x + a.y * zz.y;
          }
          if (!(l & 1)) {
            int e = (l / 2) * (l + 1) + l / 2;
            double2 a = vpart[hb + e], zz = zs[z0 + e];
            s += 0.5 * (a.x * zz.x + a.y * zz.y);
          }
          tot += d.fac[term] * s;
        }
        gacc[(size_t)si * K + b] += 2.0 * tot + io.gE * bs[b];
      }
      __syncthreads();
    }
  }
  if (MODE == MODE_VJP) {
    __syncthreads();
    for (int q = threadIdx.x; q < S.nsp * K; q += blockDim.x) io.gpart[(size_t)blockIdx.x * S.nsp * K + q] = gacc[q];
  }
}

// ---- exact Hessian-vector product (second-order adjoint) ------------------------------------
// The position pullback of the forces needs H v (H: the Hessian of E, v: the force cotangent).
// It is the directional derivative of the adjoint force computation along dx = v: every
// quantity q of it is carried with its tangent dq/de of x + e v (forward mode over the
// reverse-mode forces), so the pair terms come out as G_ij = dE_i/dr_ij and its tangent.
//   r_ij = x_j - x_i                        tangent v_j - v_i
//   U_ij and dU_ij/dr (Wigner recursion)    recursion of the tangents (product rule, below)
//   Utot_i = sum_j sfac_j w_j U_ij          tangent by the product rule
//   Z, Y (bilinear in Utot)                 Zdot = sum cg cg (Udot U + U Udot), Ydot = Y(Zdot)
//   G_ij = 2 sum_h w_h Re(conj(D_h) Y_h)    Gdot = 2 sum w Re(conj(Ddot) Y + conj(D) Ydot),
//                                           D_k = dsfac u_k U + sfac dU_k
// The tangent of the forces is the same gather of Gdot as the forces are of G, and
// H v = -Fdot.  Design: the second-order extension of compute_dij.jl:5-74 (dE/dr from dU and
// Y); one block per atom, as k_snap_atom.

// A number with its tangent.
struct Dual {
  double v, t;
};
__device__ __forceinline__ Dual dd(double v, double t = 0.0) { return Dual{v, t}; }
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual{a.v + b.v, a.t + b.t}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual{a.v - b.v, a.t - b.t}; }
__device__ __forceinline__ Dual operator-(Dual a) { return Dual{-a.v, -a.t}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual{a.v * b.v, a.t * b.v + a.v * b.t}; }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return Dual{a * b.v, a * b.t}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
  const double q = a.v / b.v;
  return Dual{q, (a.t - q * b.t) / b.v};
}
__device__ __forceinline__ Dual dsqrt(Dual a) {
  const double r = sqrt(a.v);
  return Dual{r, a.t / (2.0 * r)};
}

// The pair geometry of geom_du with tangents along (tx, ty, tz) = dr/de.
struct PairGeomD {
  Dual ar, ai, br, bi;            // a, b
  Dual dar[3], dai[3], dbr[3], dbi[3];  // da/dr_k, db/dr_k
  Dual u[3];                      // r / |r|
  Dual sfac, dsfac;               // switching function (times the neighbor weight) and its r-derivative
};

__device__ __forceinline__ void geom_hvp(const SnapDev& S, double x, double y, double z, double tx, double ty,
                                         double tz, double rcut, double wj, PairGeomD& G) {
  const Dual X = dd(x, tx), Y = dd(y, ty), Zc = dd(z, tz);
  const Dual rsq = X * X + Y * Y + Zc * Zc;
  const Dual r = dsqrt(rsq);
  const double rscale0 = S.rfac0 * M_PI / (rcut - S.rmin0);
  const Dual theta0 = rscale0 * (r - dd(S.rmin0));
  double sn, cs;
  sincos(theta0.v, &sn, &cs);
  const Dual Sn = dd(sn, cs * theta0.t), Cs = dd(cs, -sn * theta0.t);
  const Dual z0 = r * Cs / Sn;
  const Dual dz0dr = z0 / r - (rscale0 * r) * (rsq + z0 * z0) / rsq;
  const Dual rinv = dd(1.0) / r;
  G.u[0] = X * rinv;
  G.u[1] = Y * rinv;
  G.u[2] = Zc * rinv;
  const Dual r0inv = dd(1.0) / dsqrt(r * r + z0 * z0);
  G.ar = z0 * r0inv;
  G.ai = -(Zc * r0inv);
  G.br = Y * r0inv;
  G.bi = -(X * r0inv);
  const Dual dr0invdr = -(r0inv * r0inv * r0inv * (r + z0 * dz0dr));
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const Dual dr0 = dr0invdr * G.u[k];
    const Dual dz0 = dz0dr * G.u[k];
    G.dar[k] = dz0 * r0inv + z0 * dr0;
    G.dai[k] = -(Zc * dr0);
    G.dbr[k] = Y * dr0;
    G.dbi[k] = -(X * dr0);
  }
  G.dai[2] = G.dai[2] - r0inv;
  G.dbi[0] = G.dbi[0] - r0inv;
  G.dbr[1] = G.dbr[1] + r0inv;
  // compute_sfac / compute_dsfac (compute_ui.jl:350-380, the branches of sfac_of and
  // dsfac_of) with tangents
  if (!S.switch_flag || r.v <= S.rmin0) {
    G.sfac = dd(wj);
    G.dsfac = dd(0.0);
  } else {
    const double rcutfac = M_PI / (rcut - S.rmin0);
    double s2, c2;
    sincos((r.v - S.rmin0) * rcutfac, &s2, &c2);
    const double rt = r.t * rcutfac;
    G.sfac = r.v > rcut ? dd(0.0) : dd(wj * (0.5 * (c2 + 1.0)), wj * (-0.5 * s2 * rt));
    G.dsfac = dd(wj * (-0.5 * (s2 * rcutfac)), wj * (-0.5 * c2 * rcutfac * rt));
  }
}

// conj(p) * v for complex p = (pr, pi) and v, accumulated with weight c into acc.
__device__ __forceinline__ void cj_acc(double pr, double pi, double2 v, double c, double2& acc) {
  acc.x += c * (pr * v.x + pi * v.y);
  acc.y += c * (pr * v.y - pi * v.x);
}

// One level of the recursion for the eight components [U, dU/dr_k, Udot, (dU/dr_k)dot] of one
// pair, lanes over (component, entry); buffers [8][ext_max] (layout of wigner_level).
//   U_j      = f(a, b, U)
//   dU_k,j   = f(da_k, db_k, U) + f(a, b, dU_k)
//   Udot_j   = f(adot, bdot, U) + f(a, b, Udot)
//   dUdot_k  = f(da_k dot, db_k dot, U) + f(da_k, db_k, Udot) + f(adot, bdot, dU_k) + f(a, b, dUdot_k)
// with f(A, B, u)[mb][ma] = -rootpq[ma][j-mb] conj(B) u[mb][ma-1] + rootpq[j-ma][j-mb] conj(A) u[mb][ma].
// values_only: the two components U and Udot (Utot needs no derivative), else all eight.
__device__ __forceinline__ void wigner_level_hvp(const SnapDev& S, const double* rpq, int j, const PairGeomD& G,
                                                 const double2* __restrict__ prev, double2* __restrict__ cur,
                                                 int lane, bool values_only) {
  const int J2 = S.J + 2;
  const int em = S.ext_max;
  const int nrec = (j / 2 + 1) * (j + 1);
  const int ncomp = values_only ? 2 : 8;
  for (int t = lane; t < ncomp * nrec; t += 32) {
    const int grp = t / nrec;  // component group: U, Udot (values_only) or all eight
    const int comp = values_only ? grp * 4 : grp;
    const int e = t - grp * nrec;
    const int mb = e / (j + 1);
    const int ma = e - mb * (j + 1);
    const int k = (comp & 3) - 1;  // derivative direction of comps 1..3 and 5..7
    const bool tangent = comp >= 4;
    double2 res = make_double2(0.0, 0.0);
    for (int side = 0; side < 2; side++) {  // side 0: the b term at ma-1; side 1: the a term at ma
      if (side == 0 && ma == 0) continue;
      if (side == 1 && ma == j) continue;
      const int src = side == 0 ? mb * j + ma - 1 : mb * j + ma;
      const double rp = side == 0 ? -rpq[ma * J2 + (j - mb)] : rpq[(j - ma) * J2 + (j - mb)];
      const Dual pr = side == 0 ? G.br : G.ar, pi = side == 0 ? G.bi : G.ai;
      double2 acc = make_double2(0.0, 0.0);
      // f(a, b, own component)
      cj_acc(pr.v, pi.v, prev[comp * em + src], 1.0, acc);
      if (k >= 0) {  // f(da_k, db_k, U): the geometry derivative times U (and its tangent part)
        const Dual qr = side == 0 ? G.dbr[k] : G.dar[k], qi = side == 0 ? G.dbi[k] : G.dai[k];
        cj_acc(qr.v, qi.v, prev[(tangent ? 4 : 0) * em + src], 1.0, acc);
        if (tangent) {
          cj_acc(qr.t, qi.t, prev[src], 1.0, acc);        // (da_k dot) U
          cj_acc(pr.t, pi.t, prev[(k + 1) * em + src], 1.0, acc);  // adot dU_k
        }
      } else if (tangent) {  // Udot: f(adot, bdot, U)
        cj_acc(pr.t, pi.t, prev[src], 1.0, acc);
      }
      res.x += rp * acc.x;
      res.y += rp * acc.y;
    }
    cur[comp * em + e] = res;
  }
  __syncwarp();
  if (j & 1) {  // mirrored row R = (j+1)/2 of every component (inversion symmetry)
    const int R = (j + 1) / 2;
    for (int t = lane; t < ncomp * (j + 1); t += 32) {
      const int grp = t / (j + 1);
      const int comp = values_only ? grp * 4 : grp;
      const int c = t - grp * (j + 1);
      const double2 src = cur[comp * em + (j - R) * (j + 1) + (j - c)];
      const double sg = ((c + R) & 1) ? -1.0 : 1.0;
      cur[comp * em + R * (j + 1) + c] = make_double2(sg * src.x, -sg * src.y);
    }
    __syncwarp();
  }
}

// Shared memory of k_snap_hvp (doubles): Utot and its tangent [2][idxu_max] complex, the
// per-warp partial sums of both [2][nwarps][u_half] complex (aliasing Z), Z and Zdot
// [2][idxz_max] complex, Y and Ydot [2][u_half] complex, sqrt(p/q), the per-warp level
// buffers [nwarps][2 levels][8][ext_max] complex.
struct HvpSmem {
  size_t ut, zs, ys, rpq, lv, total;
};
__host__ __device__ inline HvpSmem hvp_smem(const SnapDev& S, int nwarps) {
  HvpSmem L;
  size_t o = 0;
  L.ut = o;
  o += al16(4 * (size_t)S.idxu_max);
  L.zs = o;
  const size_t zsz = 4 * (size_t)S.idxz_max, usz = 4 * (size_t)nwarps * S.u_half;
  o += al16(zsz > usz ? zsz : usz);
  L.ys = o;
  o += al16(4 * (size_t)S.u_half);
  L.rpq = o;
  o += al16((size_t)(S.J + 2) * (S.J + 2));
  L.lv = o;
  o += al16((size_t)nwarps * 2 * 8 * 2 * S.ext_max);
  L.total = o * sizeof(double);
  return L;
}

// Per pair p = (i, j): fvec[p] = dE_i/dr_ij and fdot[p] = its tangent along the atom
// displacements v [n][3].  Inputs as k_snap_atom<MODE_ADJ> (beta via S.ycoef).
__global__ void __launch_bounds__(256) k_snap_hvp(const __grid_constant__ SnapDev S, SnapIO io,
                                                  const double* __restrict__ v, double* __restrict__ fdot) {
  extern __shared__ double smem[];
  const int nwarps = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const HvpSmem L = hvp_smem(S, nwarps);
  double2* ut = reinterpret_cast<double2*>(smem + L.ut);  // [2][idxu_max]: Utot, Utot dot
  double2* utd = ut + S.idxu_max;
  double2* zs = reinterpret_cast<double2*>(smem + L.zs);  // [2][idxz_max]
  double2* zsd = zs + S.idxz_max;
  double2* ys = reinterpret_cast<double2*>(smem + L.ys);  // [2][u_half]
  double2* ysd = ys + S.u_half;
  double* rpq = smem + L.rpq;
  const int em = S.ext_max;
  double2* lv0 = reinterpret_cast<double2*>(smem + L.lv) + (size_t)warp * 2 * 8 * em;
  double2* lv1 = lv0 + 8 * em;
  const int J = S.J, uh = S.u_half;
  for (int q = threadIdx.x; q < (J + 2) * (J + 2); q += blockDim.x) rpq[q] = S.rootpq[q];
  __syncthreads();
  for (int64_t i = blockIdx.x; i < io.n; i += gridDim.x) {
    const int64_t beg = io.off[i], end = io.off[i + 1];
    const int si = clamp_sp(io.species[i], S.nsp);
    const double vi[3] = {v[3 * i], v[3 * i + 1], v[3 * i + 2]};
    // ---- Utot and its tangent (per-warp partials, then a fixed-order sum) ----
    double2* up = zs;  // [2][nwarps][u_half]
    for (int q = threadIdx.x; q < 2 * nwarps * uh; q += blockDim.x) up[q] = make_double2(0.0, 0.0);
    __syncthreads();
    {
      double2* upw = up + (size_t)warp * uh;
      double2* updw = up + (size_t)(nwarps + warp) * uh;
      for (int64_t p = beg + warp; p < end; p += nwarps) {
        const int32_t jn = io.nbr[p];
        const int sj = clamp_sp(io.species[jn], S.nsp);
        const double rcut = (S.radii[si] + S.radii[sj]) * S.rcutfac;
        const double t3[3] = {v[3 * jn] - vi[0], v[3 * jn + 1] - vi[1], v[3 * jn + 2] - vi[2]};
        PairGeomD G;
        geom_hvp(S, io.rij[3 * p], io.rij[3 * p + 1], io.rij[3 * p + 2], t3[0], t3[1], t3[2], rcut, S.weight[sj], G);
        double2* prev = lv0;
        double2* cur = lv1;
        for (int j = 0; j <= J; j++) {
          if (j == 0) {
            if (lane < 8) cur[lane * em] = make_double2(lane == 0 ? 1.0 : 0.0, 0.0);
            __syncwarp();
          } else {
            wigner_level_hvp(S, rpq, j, G, prev, cur, lane, true);
          }
          const int nrec = (j / 2 + 1) * (j + 1);
          const int hb = S.half_block[j];
          for (int e = lane; e < nrec; e += 32) {
            const double2 u = cur[e], ud = cur[4 * em + e];
            upw[hb + e].x += G.sfac.v * u.x;
            upw[hb + e].y += G.sfac.v * u.y;
            updw[hb + e].x += G.sfac.t * u.x + G.sfac.v * ud.x;
            updw[hb + e].y += G.sfac.t * u.y + G.sfac.v * ud.y;
          }
          __syncwarp();
          double2* tmp = prev;
          prev = cur;
          cur = tmp;
        }
      }
    }
    __syncthreads();
    for (int h = threadIdx.x; h < uh; h += blockDim.x) {
      double2 s = make_double2(0.0, 0.0), sd = make_double2(0.0, 0.0);
      for (int w = 0; w < nwarps; w++) {
        const double2 a = up[(size_t)w * uh + h], b = up[(size_t)(nwarps + w) * uh + h];
        s.x += a.x;
        s.y += a.y;
        sd.x += b.x;
        sd.y += b.y;
      }
      int j = 0;
      while (j < J && S.half_block[j + 1] <= h) j++;
      const int e = h - S.half_block[j];
      const int mb = e / (j + 1), ma = e - mb * (j + 1);
      if (ma == mb) s.x += S.wself;
      const int ub = S.idxu_block[j];
      const bool middle = (2 * mb == j);
      if (middle && ma > mb) continue;
      ut[ub + mb * (j + 1) + ma] = s;
      utd[ub + mb * (j + 1) + ma] = sd;
      if (!(middle && ma == mb)) {
        const double sg = ((ma + mb) & 1) ? -1.0 : 1.0;
        ut[ub + (j - mb) * (j + 1) + (j - ma)] = make_double2(sg * s.x, -sg * s.y);
        utd[ub + (j - mb) * (j + 1) + (j - ma)] = make_double2(sg * sd.x, -sg * sd.y);
      }
    }
    __syncthreads();
    // ---- Z and its tangent ----
    for (int t = threadIdx.x; t < S.idxz_max; t += blockDim.x) {
      const int jjz = S.zperm[t];
      const ZDev q = S.idxz[jjz];
      const double* cgb = S.cglist + q.cgoff;
      const int j1 = q.j1, j2 = q.j2;
      double zr = 0.0, zi = 0.0, dr = 0.0, di = 0.0;
      int i1 = q.u1base, i2 = q.u2base, icgb = q.icgb0;
      for (int ib = 0; ib < q.nb; ib++) {
        double sr = 0.0, sim = 0.0, tr = 0.0, tim = 0.0;
        int icga = q.icga0;
        for (int ia = 0; ia < q.na; ia++) {
          const double2 u1 = ut[i1 + ia], u2 = ut[i2 - ia];
          const double2 d1 = utd[i1 + ia], d2 = utd[i2 - ia];
          const double c = __ldg(cgb + icga);
          sr += c * (u1.x * u2.x - u1.y * u2.y);
          sim += c * (u1.x * u2.y + u1.y * u2.x);
          tr += c * (d1.x * u2.x - d1.y * u2.y + u1.x * d2.x - u1.y * d2.y);
          tim += c * (d1.x * u2.y + d1.y * u2.x + u1.x * d2.y + u1.y * d2.x);
          icga += j2;
        }
        const double cb = __ldg(cgb + icgb);
        zr += cb * sr;
        zi += cb * sim;
        dr += cb * tr;
        di += cb * tim;
        i1 += j1 + 1;
        i2 -= j2 + 1;
        icgb += j2;
      }
      if (S.bnorm_flag) {
        const double f = 1.0 / (q.j + 1);
        zr *= f;
        zi *= f;
        dr *= f;
        di *= f;
      }
      zs[jjz] = make_double2(zr, zi);
      zsd[jjz] = make_double2(dr, di);
    }
    __syncthreads();
    // ---- Y and its tangent ----
    {
      const double* yc = S.ycoef + (size_t)si * S.idxz_max;
      for (int h = threadIdx.x; h < uh; h += blockDim.x) {
        double2 y = make_double2(0.0, 0.0), yd = make_double2(0.0, 0.0);
        for (int q = S.y_off[h]; q < S.y_off[h + 1]; q++) {
          const int jjz = S.y_jjz[q];
          const double c = yc[jjz];
          y.x += c * zs[jjz].x;
          y.y += c * zs[jjz].y;
          yd.x += c * zsd[jjz].x;
          yd.y += c * zsd[jjz].y;
        }
        ys[h] = y;
        ysd[h] = yd;
      }
    }
    __syncthreads();
    // ---- per neighbor: G = dE_i/dr_ij and its tangent ----
    for (int64_t p = beg + warp; p < end; p += nwarps) {
      const int32_t jn = io.nbr[p];
      const int sj = clamp_sp(io.species[jn], S.nsp);
      const double rcut = (S.radii[si] + S.radii[sj]) * S.rcutfac;
      const double t3[3] = {v[3 * jn] - vi[0], v[3 * jn + 1] - vi[1], v[3 * jn + 2] - vi[2]};
      PairGeomD G;
      geom_hvp(S, io.rij[3 * p], io.rij[3 * p + 1], io.rij[3 * p + 2], t3[0], t3[1], t3[2], rcut, S.weight[sj], G);
      double acc[3] = {0.0, 0.0, 0.0}, accd[3] = {0.0, 0.0, 0.0};
      double2* prev = lv0;
      double2* cur = lv1;
      for (int j = 0; j <= J; j++) {
        if (j == 0) {
          if (lane < 8) cur[lane * em] = make_double2(lane == 0 ? 1.0 : 0.0, 0.0);
          __syncwarp();
        } else {
          wigner_level_hvp(S, rpq, j, G, prev, cur, lane, false);
        }
        const int nrec = (j / 2 + 1) * (j + 1);
        const int hb = S.half_block[j];
        const int nf = nfull_of(j);
        const int emid = (j & 1) ? -1 : (j / 2) * (j + 1) + j / 2;
        for (int e = lane; e < nrec; e += 32) {
          const double w = (e < nf) ? 1.0 : (e == emid ? 0.5 : 0.0);
          if (w == 0.0) continue;
          const double2 u = cur[e], ud = cur[4 * em + e];
          const double2 Yv = ys[hb + e], Yd = ysd[hb + e];
#pragma unroll
          for (int k = 0; k < 3; k++) {
            const double2 du = cur[(k + 1) * em + e], dud = cur[(k + 5) * em + e];
            // D = dsfac u_k U + sfac dU_k and its tangent
            const double cu = G.dsfac.v * G.u[k].v, cut = G.dsfac.t * G.u[k].v + G.dsfac.v * G.u[k].t;
            const double Dx = cu * u.x + G.sfac.v * du.x, Dy = cu * u.y + G.sfac.v * du.y;
            const double Ddx = cut * u.x + cu * ud.x + G.sfac.t * du.x + G.sfac.v * dud.x;
            const double Ddy = cut * u.y + cu * ud.y + G.sfac.t * du.y + G.sfac.v * dud.y;
            acc[k] += w * (Dx * Yv.x + Dy * Yv.y);
            accd[k] += w * (Ddx * Yv.x + Ddy * Yv.y + Dx * Yd.x + Dy * Yd.y);
          }
        }
        __syncwarp();
        double2* tmp = prev;
        prev = cur;
        cur = tmp;
      }
#pragma unroll
      for (int k = 0; k < 3; k++) {
        acc[k] = warp_sum(acc[k]);
        accd[k] = warp_sum(accd[k]);
      }
      if (lane == 0)
        for (int k = 0; k < 3; k++) {
          io.fvec[3 * p + k] = 2.0 * acc[k];
          fdot[3 * p + k] = 2.0 * accd[k];
        }
    }
    __syncthreads();
  }
}

// ---- explicit multi-element SNAP (chem_flag) and quadratic SNAP ---------------------------
// One block per atom, the phases of k_snap_atom resolved by element (the element of the
// neighbor for Utot, compute_ui.jl:155-175; ordered element pairs for Z, compute_z.jl:5-61;
// element triples for B and dB/dr, compute_b.jl:15-95 and :104-342), and the quadratic
// products of LAMMPS_SNAP/snap.jl:45-47 (0.5 B_k^2 and B_k B_l, l > k, after the klin linear
// components).  Z of one atom (nelem^2 idxz_max complex) lives in a block-private slice of
// global memory; the rest in shared memory.
//   B_ext [n][K] (io.B, when set) and E_i = beta[s_i] . B_ext (io.Ei, bzero already in B);
//   PLAIN: dB_lin/dr of every pair, io.dbl [np][klin][3]; with quadratic_flag also the linear
//   coefficients with the same forces, beff [n][klin] (beta_k + sum_l a_kl B_l).
struct ChemSmem {
  size_t ut, up, bs, bf, rpq, lv, duf, red, total;
};
__host__ __device__ inline ChemSmem chem_smem(const SnapDev& S, int nwarps, bool plain) {
  ChemSmem L;
  size_t o = 0;
  L.ut = o;
  o += al16(2 * (size_t)S.nelem * S.idxu_max);
  L.up = o;  // per-warp partial Utot [nwarps][nelem][u_half]
  o += al16(2 * (size_t)nwarps * S.nelem * S.u_half);
  L.bs = o;  // linear B [klin]
  o += al16((size_t)S.klin);
  L.bf = o;  // effective linear coefficients [klin]
  o += al16((size_t)S.klin);
  L.rpq = o;
  o += al16((size_t)(S.J + 2) * (S.J + 2));
  L.lv = o;
  o += al16((size_t)nwarps * 2 * 4 * 2 * S.ext_max);
  L.duf = o;
  if (plain) o += al16((size_t)nwarps * 2 * 3 * S.u_half);
  L.red = o;
  o += al16(256);
  L.total = o * sizeof(double);
  return L;
}

// First slot of row k of the quadratic block: Klin + sum_{q<k} (Klin - q).
__device__ __forceinline__ int quad_row(int klin, int k) { return klin + k * klin - k * (k - 1) / 2; }

template <bool PLAIN>
__global__ void __launch_bounds__(128) k_snap_chem(const __grid_constant__ SnapDev S, SnapIO io,
                                                   double2* __restrict__ zbuf, double* __restrict__ beff) {
  extern __shared__ double smem[];
  const int nwarps = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const ChemSmem L = chem_smem(S, nwarps, PLAIN);
  double2* ut = reinterpret_cast<double2*>(smem + L.ut);  // [nelem][idxu_max]
  double2* upart = reinterpret_cast<double2*>(smem + L.up);
  double* bs = smem + L.bs;
  double* bfe = smem + L.bf;
  double* rpq = smem + L.rpq;
  double* red = smem + L.red;
  double2* lv0 = reinterpret_cast<double2*>(smem + L.lv) + (size_t)warp * 2 * 4 * S.ext_max;
  double2* lv1 = lv0 + 4 * S.ext_max;
  const int J = S.J, K = S.K, KL = S.klin, uh = S.u_half, U = S.idxu_max, M = S.idxz_max;
  const int ne = S.nelem, KB = KL / (ne * ne * ne);  // components per element triple (idxb_max)
  double2* zb = zbuf + (size_t)blockIdx.x * ne * ne * M;
  for (int q = threadIdx.x; q < (J + 2) * (J + 2); q += blockDim.x) rpq[q] = S.rootpq[q];
  __syncthreads();
  for (int64_t i = blockIdx.x; i < io.n; i += gridDim.x) {
    const int64_t beg = io.off[i], end = io.off[i + 1];
    const int si = clamp_sp(io.species[i], S.nsp);
    const int ielem = S.chem ? si : 0;
    // ---- Utot of every element ----
    for (int q = threadIdx.x; q < nwarps * ne * uh; q += blockDim.x) upart[q] = make_double2(0.0, 0.0);
    __syncthreads();
    for (int64_t p = beg + warp; p < end; p += nwarps) {
      const double x = io.rij[3 * p], y = io.rij[3 * p + 1], z = io.rij[3 * p + 2];
      const int sj = clamp_sp(io.species[io.nbr[p]], S.nsp);
      const double rcut = (S.radii[si] + S.radii[sj]) * S.rcutfac;
      const double r = sqrt(x * x + y * y + z * z);
      const double theta0 = (r - S.rmin0) * S.rfac0 * M_PI / (rcut - S.rmin0);
      const double z0 = r / tan(theta0);
      const double r0inv = 1.0 / sqrt(r * r + z0 * z0);
      PairGeom G;
      G.a = make_double2(r0inv * z0, -r0inv * z);
      G.b = make_double2(r0inv * y, -r0inv * x);
      const double sw = sfac_of(S, r, rcut) * S.weight[sj];
      double2* up = upart + ((size_t)warp * ne + (S.chem ? sj : 0)) * uh;
      double2* prev = lv0;
      double2* cur = lv1;
      if (lane == 0) {
        prev[0] = make_double2(1.0, 0.0);
        up[0].x += sw;
      }
      __syncwarp();
      for (int j = 1; j <= J; j++) {
        wigner_level(S, rpq, j, 1, G, prev, cur, lane);
        const int nrec = (j / 2 + 1) * (j + 1);
        double2* upj = up + S.half_block[j];
        for (int e = lane; e < nrec; e += 32) {
          upj[e].x += sw * cur[e].x;
          upj[e].y += sw * cur[e].y;
        }
        __syncwarp();
        double2* t = prev;
        prev = cur;
        cur = t;
      }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < ne * uh; t += blockDim.x) {
      const int el = t / uh, h = t - el * uh;
      double2 sacc = make_double2(0.0, 0.0);
      for (int w = 0; w < nwarps; w++) {
        const double2 v = upart[((size_t)w * ne + el) * uh + h];
        sacc.x += v.x;
        sacc.y += v.y;
      }
      int j = 0;
      while (j < J && S.half_block[j + 1] <= h) j++;
      const int e = h - S.half_block[j];
      const int mb = e / (j + 1), ma = e - mb * (j + 1);
      if (ma == mb && (el == ielem || S.wselfall)) sacc.x += S.wself;  // zero_uarraytot
      const int ub = el * U + S.idxu_block[j];
      const bool middle = (2 * mb == j);
      if (middle && ma > mb) continue;
      ut[ub + mb * (j + 1) + ma] = sacc;
      if (!(middle && ma == mb)) {
        const double sg = ((ma + mb) & 1) ? -1.0 : 1.0;
        ut[ub + (j - mb) * (j + 1) + (j - ma)] = make_double2(sg * sacc.x, -sg * sacc.y);
      }
    }
    __syncthreads();
    // ---- Z of every ordered element pair (literal_chem_z: compute_z.jl's own indexing) ----
    for (int jjz = threadIdx.x; jjz < M; jjz += blockDim.x) {
      const ZDev q = S.idxz[jjz];
      const double* cgb = S.cglist + q.cgoff;
      const int j1 = q.j1, j2 = q.j2;
      for (int d = 1; d < ne * ne; d++) zb[(size_t)d * M + jjz] = make_double2(0.0, 0.0);
      double2 run = make_double2(0.0, 0.0);
      for (int d = 0; d < ne * ne; d++) {
        const double2* u1 = ut + (d / ne) * U;
        const double2* u2 = ut + (d % ne) * U;
        double zr = S.literal_chem_z ? run.x : 0.0, zi = S.literal_chem_z ? run.y : 0.0;
        int i1 = q.u1base, i2 = q.u2base, icgb = q.icgb0;
        for (int ib = 0; ib < q.nb; ib++) {
          double sr = 0.0, sim = 0.0;
          int icga = q.icga0;
          for (int ia = 0; ia < q.na; ia++) {
            const double2 a1 = u1[i1 + ia], a2 = u2[i2 - ia];
            const double c = __ldg(cgb + icga);
            sr += c * (a1.x * a2.x - a1.y * a2.y);
            sim += c * (a1.x * a2.y + a1.y * a2.x);
            icga += j2;
          }
          const double cb = __ldg(cgb + icgb);
          zr += cb * sr;
          zi += cb * sim;
          i1 += j1 + 1;
          i2 -= j2 + 1;
          icgb += j2;
        }
        if (S.bnorm_flag) {
          zr /= (q.j + 1);
          zi /= (q.j + 1);
        }
        run = make_double2(zr, zi);
        if (!S.literal_chem_z) zb[(size_t)d * M + jjz] = run;
      }
      if (S.literal_chem_z) zb[jjz] = run;
    }
    __syncthreads();
    // ---- B of every element triple ----
    for (int t = threadIdx.x; t < KL; t += blockDim.x) {
      const int tri = t / KB, b = t - tri * KB;
      const int e3 = tri % ne, d = tri / ne;  // tri = (e1 ne + e2) ne + e3, d = e1 ne + e2
      const DBDev db = S.db[b];
      const int l = db.l[0], u0 = e3 * U + S.idxu_block[l];
      const double2* zz = zb + (size_t)d * M + db.z0[0];
      const int nf = nfull_of(l);
      double sacc = 0.0;
      for (int e = 0; e < nf; e++) sacc += ut[u0 + e].x * zz[e].x + ut[u0 + e].y * zz[e].y;
      if (!(l & 1)) {
        const int e = (l / 2) * (l + 1) + l / 2;
        sacc += 0.5 * (ut[u0 + e].x * zz[e].x + ut[u0 + e].y * zz[e].y);
      }
      double Bv = 2.0 * sacc;
      if (S.bzero_flag && (S.wselfall || tri == (ielem * ne + ielem) * ne + ielem)) Bv -= S.bzero[l];
      bs[t] = Bv;
    }
    __syncthreads();
    // ---- B_ext, E_i and the effective linear coefficients ----
    const double* bt = S.beta + (size_t)si * K;
    double e = 0.0;
    for (int k = threadIdx.x; k < KL; k += blockDim.x) {
      const double bk = bs[k];
      e += bt[k] * bk;
      if (io.B) io.B[i * K + k] = bk;
      if (S.quadratic) {
        const int r0 = quad_row(KL, k);
        double g = bt[k] + bt[r0] * bk;  // d/dB_k of beta . B_ext
        const double q0 = 0.5 * bk * bk;
        e += bt[r0] * q0;
        if (io.B) io.B[i * K + r0] = q0;
        for (int l = k + 1; l < KL; l++) {
          const double q = bk * bs[l];
          e += bt[r0 + l - k] * q;
          if (io.B) io.B[i * K + r0 + l - k] = q;
          g += bt[r0 + l - k] * bs[l];
        }
        for (int l = 0; l < k; l++) g += bt[quad_row(KL, l) + k - l] * bs[l];
        bfe[k] = g;
        if (beff) beff[i * KL + k] = g;
      }
    }
    red[threadIdx.x] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < (int)blockDim.x; w++) t += red[w];
      io.Ei[i] = t;
    }
    if (PLAIN) {
      // ---- per neighbor: dB_lin/dr of every element triple (compute_b.jl:104-342) ----
      double2* dufw = reinterpret_cast<double2*>(smem + L.duf) + (size_t)warp * 3 * uh;  // [3][u_half]
      for (int64_t p = beg + warp; p < end; p += nwarps) {
        const int32_t jn = io.nbr[p];
        const int sj = clamp_sp(io.species[jn], S.nsp);
        const int e3 = S.chem ? sj : 0;
        const double rcut = (S.radii[si] + S.radii[sj]) * S.rcutfac;
        PairGeom G;
        geom_du(S, io.rij[3 * p], io.rij[3 * p + 1], io.rij[3 * p + 2], rcut, S.weight[sj], G);
        double2* prev = lv0;
        double2* cur = lv1;
        const int em = S.ext_max;
        for (int j = 0; j <= J; j++) {
          if (j == 0) {
            if (lane < 4) cur[lane * em] = make_double2(lane == 0 ? 1.0 : 0.0, 0.0);
            __syncwarp();
          } else {
            wigner_level(S, rpq, j, 4, G, prev, cur, lane);
          }
          const int nrec = (j / 2 + 1) * (j + 1);
          const int hb = S.half_block[j];
          for (int ee = lane; ee < nrec; ee += 32) {
            const double2 u = cur[ee];
#pragma unroll
            for (int k = 0; k < 3; k++) {
              const double2 dd = cur[(k + 1) * em + ee];
              dufw[k * uh + hb + ee] = make_double2(G.dsfac * u.x * G.u[k] + G.sfac * dd.x,
                                                    G.dsfac * u.y * G.u[k] + G.sfac * dd.y);
            }
          }
          __syncwarp();
          double2* t = prev;
          prev = cur;
          cur = t;
        }
        double* out = io.dbl + (size_t)p * KL * 3;
        for (int t = lane; t < 3 * KL; t += 32) {
          const int q = t / 3, k = t - 3 * q;
          const int tri = q / KB, b = q - tri * KB;
          const int c3 = tri % ne, b3 = (tri / ne) % ne, a3 = tri / (ne * ne);
          // the terms that land on triple (a3, b3, c3): term 0 with e3 = c3 and Z(a3, b3),
          // term 1 with e3 = a3 and Z(c3, b3), term 2 with e3 = b3 and Z(c3, a3)
          const int cond[3] = {c3 == e3, a3 == e3, b3 == e3};
          const int zd[3] = {a3 * ne + b3, c3 * ne + b3, c3 * ne + a3};
          const DBDev db = S.db[b];
          double tot = 0.0;
#pragma unroll
          for (int term = 0; term < 3; term++) {
            if (!cond[term]) continue;
            const int l = db.l[term], hb = S.half_block[l];
            const int nf = nfull_of(l);
            const double2* du = dufw + k * uh + hb;
            const double2* zz = zb + (size_t)zd[term] * M + db.z0[term];
            double sacc = 0.0;
            for (int ee = 0; ee < nf; ee++) sacc += du[ee].x * zz[ee].x + du[ee].y * zz[ee].y;
            if (!(l & 1)) {
              const int ee = (l / 2) * (l + 1) + l / 2;
              sacc += 0.5 * (du[ee].x * zz[ee].x + du[ee].y * zz[ee].y);
            }
            tot += db.fac[term] * sacc;
          }
          out[t] = 2.0 * tot;
        }
        __syncwarp();
      }
    }
    __syncthreads();
  }
}

// Quadratic SNAP: the per-pair dB_ext/dr [np][K][3] of the pair's centre i = owner[p] from its
// linear dB/dr [np][klin][3] and B_ext [n][K] (its first klin entries):
// d(0.5 B_k^2) = B_k dB_k, d(B_k B_l) = B_l dB_k + B_k dB_l.  Thread per (pair, component k).
__global__ void k_quad_pairs(int64_t np_cap, const int64_t* __restrict__ d_np, int klin, int K,
                             const int32_t* __restrict__ owner, const double* __restrict__ Bx,
                             const double* __restrict__ dbl, double* __restrict__ dbx) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t p = t / klin;
  const int k = (int)(t - p * klin);
  if (p >= np_cap || p >= *d_np) return;
  const double* b = Bx + (size_t)owner[p] * K;
  const double* d = dbl + (size_t)p * klin * 3;
  double* o = dbx + (size_t)p * K * 3;
  const double bk = b[k];
  for (int c = 0; c < 3; c++) o[3 * k + c] = d[3 * k + c];
  const int r0 = klin + k * klin - k * (k - 1) / 2;
  for (int c = 0; c < 3; c++) o[3 * r0 + c] = bk * d[3 * k + c];
  for (int l = k + 1; l < klin; l++)
    for (int c = 0; c < 3; c++) o[3 * (r0 + l - k) + c] = b[l] * d[3 * k + c] + bk * d[3 * l + c];
}

// Utot of every atom (compute_ui.jl:5-175) from the register chains: one launch per
// chain MB, one warp per atom, lanes over neighbors (32 at a time).  Each chain's rows
// (and their mirrors) are disjoint, so the launches write disjoint entries of
// utot[i][idxu_max]; the per-entry sums over lanes are warp reductions in fixed order.
template <int J, int MB>
__global__ void __launch_bounds__(128) k_snap_utot(const __grid_constant__ SnapDev S, int64_t n,
                                                  const int64_t* __restrict__ off, const int32_t* __restrict__ nbr,
                                                  const double* __restrict__ rij,
                                                  const int32_t* __restrict__ species, double2* __restrict__ utot) {
  const int lane = threadIdx.x & 31;
  const int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (i >= n) return;  // warp-uniform
  const int si = clamp_sp(species[i], S.nsp);
  const int64_t beg = off[i], end = off[i + 1];
  double2* ut = utot + (size_t)i * S.idxu_max;
  for (int64_t p0 = beg; p0 < (end > beg ? end : beg + 1); p0 += 32) {
    const int64_t p = p0 + lane;
    double2 a = make_double2(1.0, 0.0), b = make_double2(0.0, 0.0);
    double sw = 0.0;  // idle lanes contribute zero
    if (p < end) {
      const double x = rij[3 * p], y = rij[3 * p + 1], z = rij[3 * p + 2];
      const int sj = clamp_sp(species[nbr[p]], S.nsp);
      const double rcut = (S.radii[si] + S.radii[sj]) * S.rcutfac;  // runtime_arrays.jl:50
      const double r = sqrt(x * x + y * y + z * z);
      const double theta0 = (r - S.rmin0) * S.rfac0 * M_PI / (rcut - S.rmin0);
      const double z0 = r / tan(theta0);
      const double r0inv = 1.0 / sqrt(r * r + z0 * z0);
      a = make_double2(r0inv * z0, -r0inv * z);
      b = make_double2(r0inv * y, -r0inv * x);
      sw = sfac_of(S, r, rcut) * S.weight[sj];
    }
    snapchain::chain_utot_emit<J, MB>(a, b, sw, ut, lane, p0 == beg, S.wself);
  }
}

// Utot of every atom in one launch: one warp per atom, lanes over neighbors (32 at a time),
// every chain of a neighbor in its lane (snapchain::all_chains_utot); the sums over lanes go
// through a per-warp staging buffer in shared memory, in fixed order.
constexpr int UTA_WARPS = 4;
template <int J>
__global__ void __launch_bounds__(UTA_WARPS * 32) k_snap_utot_all(const __grid_constant__ SnapDev S, int64_t n,
                                                                  const int64_t* __restrict__ off,
                                                                  const int32_t* __restrict__ nbr,
                                                                  const double* __restrict__ rij,
                                                                  const int32_t* __restrict__ species,
                                                                  double2* __restrict__ utot) {
  __shared__ double2 buf[UTA_WARPS][snapchain::UT_SLOTS * 33];
  __shared__ int dst[UTA_WARPS][snapchain::UT_SLOTS];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t i = (int64_t)blockIdx.x * UTA_WARPS + w;
  if (i >= n) return;  // warp-uniform; the kernel synchronises only within a warp
  const int si = clamp_sp(species[i], S.nsp);
  const int64_t beg = off[i], end = off[i + 1];
  snapchain::UtStage st;
  st.buf = buf[w];
  st.dst = dst[w];
  st.ut = reinterpret_cast<double*>(utot + (size_t)i * S.idxu_max);
  st.lane = lane;
  st.nslot = 0;
  st.wself = S.wself;
  for (int64_t p0 = beg; p0 < (end > beg ? end : beg + 1); p0 += 32) {
    const int64_t p = p0 + lane;
    double2 a = make_double2(1.0, 0.0), b = make_double2(0.0, 0.0);
    double sw = 0.0;  // idle lanes contribute zero
    if (p < end) {
      const double x = rij[3 * p], y = rij[3 * p + 1], z = rij[3 * p + 2];
      const int sj = clamp_sp(species[nbr[p]], S.nsp);
      const double rcut = (S.radii[si] + S.radii[sj]) * S.rcutfac;  // runtime_arrays.jl:50
      const double r = sqrt(x * x + y * y + z * z);
      const double theta0 = (r - S.rmin0) * S.rfac0 * M_PI / (rcut - S.rmin0);
      const double z0 = r / tan(theta0);
      const double r0inv = 1.0 / sqrt(r * r + z0 * z0);
      a = make_double2(r0inv * z0, -r0inv * z);
      b = make_double2(r0inv * y, -r0inv * x);
      sw = sfac_of(S, r, rcut) * S.weight[sj];
    }
    st.first = p0 == beg;
    snapchain::all_chains_utot<J>(a, b, sw, st);
  }
}

template <int J>
int launch_utot_all(ipg_ctx* ctx, const SnapDev& S, int64_t n, const int64_t* off, const int32_t* nbr,
                    const double* rij, const int32_t* species, double2* utot) {
  IPG_TIMED_LAUNCH(ctx, "snap_utot", k_snap_utot_all<J>, nblk(n, UTA_WARPS), UTA_WARPS * 32, 0, S, n, off, nbr, rij,
                   species, utot);
  return IPG_OK;
}

template <int J, int MB>
int launch_utot_chains(ipg_ctx* ctx, const SnapDev& S, int64_t n, const int64_t* off, const int32_t* nbr,
                       const double* rij, const int32_t* species, double2* utot, int warps) {
  if constexpr (MB <= J / 2) {
    IPG_TIMED_LAUNCH(ctx, "snap_utot", (k_snap_utot<J, MB>), nblk(n, warps), 32 * warps, 0, S, n, off, nbr, rij,
                     species, utot);
    return launch_utot_chains<J, MB + 1>(ctx, S, n, off, nbr, rij, species, utot, warps);
  }
  return IPG_OK;
}

// warps: atoms (warps) per block, 1..4, of the per-chain kernels; all_chains: one launch of
// k_snap_utot_all instead.
int launch_utot(ipg_ctx* ctx, const SnapDev& S, int64_t n, const int64_t* off, const int32_t* nbr,
                const double* rij, const int32_t* species, double2* utot, int warps = 4, bool all_chains = true) {
  if (n == 0) return IPG_OK;
  warps = std::max(1, std::min(4, warps));
  if (all_chains) {
    switch (S.J) {
#define IPG_J(JJ) \
  case JJ:        \
    return launch_utot_all<JJ>(ctx, S, n, off, nbr, rij, species, utot);
      IPG_J(0) IPG_J(1) IPG_J(2) IPG_J(3) IPG_J(4) IPG_J(5) IPG_J(6) IPG_J(7) IPG_J(8) IPG_J(9) IPG_J(10)
#undef IPG_J
      default:
        return IPG_ERR_UNSUPPORTED;
    }
  }
  switch (S.J) {
#define IPG_J(JJ) \
  case JJ:        \
    return launch_utot_chains<JJ, 0>(ctx, S, n, off, nbr, rij, species, utot, warps);
    IPG_J(0) IPG_J(1) IPG_J(2) IPG_J(3) IPG_J(4) IPG_J(5) IPG_J(6) IPG_J(7) IPG_J(8) IPG_J(9) IPG_J(10)
#undef IPG_J
    default:
      return IPG_ERR_UNSUPPORTED;
  }
}


// The inner CG sum of one ib for the calling lane's atom: sum_ia ca[ia] u1[ia] u2[ia]
// with u1 = U(j1, mb1, ma1min + ia) and u2 = U(j2, mb2, ma2max - ia).  Only rows
// mb <= j/2 are stored (the half plane, [h][atom]); a row beyond it is read from its
// mirror, U[j][mb][ma] = (-1)^(ma+mb) conj(U[j][j-mb][j-ma]) (compute_ui.jl:105-125):
// its sign alternates with ia (folded into the FMAs) and its conjugate flips the sign of
// the imaginary part.  M1, M2 say which of the two rows is mirrored.
template <int NA, bool M1, bool M2>
__device__ __forceinline__ void zrow_lanes(const double* ca, const double2* __restrict__ p1,
                                           const double2* __restrict__ p2, double& sr, double& sim) {
  constexpr int d1 = M1 ? -YS_ATOMS : YS_ATOMS;  // step of ma1 in storage
  constexpr int d2 = M2 ? YS_ATOMS : -YS_ATOMS;  // step of ma2 in storage
#pragma unroll
  for (int ia = 0; ia < NA; ia++) {
    const double2 v1 = p1[ia * d1];
    const double2 v2 = p2[ia * d2];
    const double u1y = M1 ? -v1.y : v1.y;
    const double u2y = M2 ? -v2.y : v2.y;
    // alternating sign of a single mirrored row; two mirrored rows: signs cancel per ia
    const double c = (M1 != M2 && (ia & 1)) ? -ca[ia] : ca[ia];
    sr += c * (v1.x * v2.x - u1y * u2y);
    sim += c * (v1.x * u2y + u1y * v2.x);
  }
}

// One Z entry (compute_z.jl:8-57) for the calling lane's atom, na a compile-time
// constant.  The na CG factors of the inner sum are the same for every ib (icga restarts
// at icga0), so they are loaded once.
template <int NA>
__device__ __forceinline__ double2 zitem_lanes(const ZDev& z, const double* __restrict__ cgb,
                                               const double2* __restrict__ uh, const int* __restrict__ hblk,
                                               int mb1min, int ma1min, int mb2max, int ma2max) {
  double ca[NA];
#pragma unroll
  for (int ia = 0; ia < NA; ia++) ca[ia] = __ldg(cgb + z.icga0 + ia * z.j2);
  const int j1 = z.j1, j2 = z.j2;
  double zr = 0.0, zi = 0.0;
  int icgb = z.icgb0;
  for (int ib = 0; ib < z.nb; ib++) {
    const int mb1 = mb1min + ib, mb2 = mb2max - ib;
    const bool m1 = 2 * mb1 > j1, m2 = 2 * mb2 > j2;
    const int r1 = m1 ? j1 - mb1 : mb1, c1 = m1 ? j1 - ma1min : ma1min;
    const int r2 = m2 ? j2 - mb2 : mb2, c2 = m2 ? j2 - ma2max : ma2max;
    const double2* p1 = uh + (size_t)(hblk[j1] + r1 * (j1 + 1) + c1) * YS_ATOMS;
    const double2* p2 = uh + (size_t)(hblk[j2] + r2 * (j2 + 1) + c2) * YS_ATOMS;
    double sr = 0.0, sim = 0.0;
    if (!m1 && !m2) zrow_lanes<NA, false, false>(ca, p1, p2, sr, sim);
    else if (m1 && !m2) zrow_lanes<NA, true, false>(ca, p1, p2, sr, sim);
    else if (!m1 && m2) zrow_lanes<NA, false, true>(ca, p1, p2, sr, sim);
    else zrow_lanes<NA, true, true>(ca, p1, p2, sr, sim);
    // sign of the ia = 0 term of the mirrored row(s): (-1)^(ma+mb)
    const int par = (m1 ? (ma1min + mb1) : 0) + (m2 ? (ma2max + mb2) : 0);
    const double cb = (par & 1) ? -__ldg(cgb + icgb) : __ldg(cgb + icgb);
    zr += cb * sr;
    zi += cb * sim;
    icgb += j2;
  }
  return make_double2(zr, zi);
}

// Adjoint per-atom part, "atoms in lanes": a block takes YS_ATOMS atoms, keeps their
// Utot in shared memory as [entry][atom] and every lane walks the same Z entries for its
// own atom, so table and Clebsch-Gordan loads are warp-uniform broadcasts and the Utot
// reads are conflict-free.  Warp w owns a cost-balanced set of half-plane entries h and
// accumulates Y_h = sum_{Z entries of h} coef * Z in registers (design of
// compute_yi.jl:23-121), then writes Y'_h = w_h Y_h to yout[h][atom] and adds
// Re(conj(U_h) Y'_h) to the atom's energy: E_i = (2/3) sum_h Re(conj(U_h) Y'_h) - beta.bzero
// (B is cubic in U).
static_assert(SNAP_MAX_J + 1 <= 13, "k_snap_yatoms covers Z entries of up to 13 terms");
__global__ void __launch_bounds__(YS_WARPS * 32, 2) k_snap_yatoms(const __grid_constant__ SnapDev S, int64_t n,
                                                                  const int32_t* __restrict__ species,
                                                                  const double2* __restrict__ utot,
                                                                  double2* __restrict__ yout, double* __restrict__ Ei) {
  extern __shared__ double2 us[];  // half plane of Utot: [u_half][YS_ATOMS]
  __shared__ double esum[YS_WARPS][YS_ATOMS];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int U = S.idxu_max, UH = S.u_half;
  for (int64_t a0 = (int64_t)blockIdx.x * YS_ATOMS; a0 < n; a0 += (int64_t)gridDim.x * YS_ATOMS) {
    const int na_blk = (int)((n - a0) < YS_ATOMS ? (n - a0) : YS_ATOMS);
    for (int idx = threadIdx.x; idx < UH * YS_ATOMS; idx += blockDim.x) {
      const int q = idx / YS_ATOMS, l = idx - q * YS_ATOMS;
      us[idx] = l < na_blk ? utot[(size_t)(a0 + l) * U + S.u_of_h[q]] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    const int64_t atom = a0 + lane;
    const bool valid = lane < na_blk;
    const int si = valid ? clamp_sp(species[atom], S.nsp) : 0;
    const double* yc = S.ycoef + (size_t)si * S.idxz_max;
    double e = 0.0;
    for (int hh = S.ysched_off[warp]; hh < S.ysched_off[warp + 1]; hh++) {
      const int h = S.ysched_h[hh];
      double yr = 0.0, yi = 0.0;
      for (int q = S.y_off[h]; q < S.y_off[h + 1]; q++) {
        const int jjz = S.y_jjz[q];
        const ZDev z = S.idxz[jjz];
        const int mb1min = z.mb1min, ma1min = z.ma1min, mb2max = z.mb2max, ma2max = z.ma2max;
        double2 zz;
        switch (z.na) {  // warp-uniform: every lane walks the same Z entry
#define IPG_NA(NA)                                                                                        \
  case NA:                                                                                                \
    zz = zitem_lanes<NA>(z, S.cglist + z.cgoff, us + lane, S.half_block, mb1min, ma1min, mb2max, ma2max); \
    break;
          // na <= j1 + 1 <= SNAP_MAX_J + 1 (j1 = j2 = twojmax, j = 0 reaches it)
          IPG_NA(1) IPG_NA(2) IPG_NA(3) IPG_NA(4) IPG_NA(5) IPG_NA(6) IPG_NA(7) IPG_NA(8) IPG_NA(9) IPG_NA(10)
          IPG_NA(11) IPG_NA(12) IPG_NA(13)
#undef IPG_NA
          default:
            zz = make_double2(0.0, 0.0);
        }
        double zr = zz.x, zi = zz.y;
        if (S.bnorm_flag) {
          zr /= (z.j + 1);
          zi /= (z.j + 1);
        }
        const double c = yc[jjz];
        yr += c * zr;
        yi += c * zi;
      }
      const double w = S.ysched_w[hh];
      yr *= w;
      yi *= w;
      if (valid) yout[(size_t)h * n + atom] = make_double2(yr, yi);
      const double2 u = us[(size_t)h * YS_ATOMS + lane];
      e += u.x * yr + u.y * yi;
    }
    esum[warp][lane] = e;
    __syncthreads();
    if (warp == 0 && valid) {
      double t = 0.0;
      for (int w = 0; w < YS_WARPS; w++) t += esum[w][lane];
      Ei[atom] = (2.0 / 3.0) * t + S.ebias[si];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------
// Row-blocked Y kernel.  Same block shape as k_snap_yatoms (32 atoms in the lanes, the
// half plane of their Utot in shared memory as [h][atom]), but a warp owns whole target
// rows (j, mb) of Y and, for each triple (j1, j2, j) feeding the row and each of its nb
// row pairs (mb1, mb2), evaluates the Z entries of every ma of the row at once:
//   Y(j, mb, ma) += c cg[mb1][mb2] sum_ma2 ca[ma][ma2] U(j1, mb1, ma + d - ma2) U(j2, mb2, ma2),
// d = (j1 + j2 - j)/2, c = the triple's Y coefficient (compute_yi.jl:86-118).  The j2 row
// is walked two columns at a time; each element of the j1 row met by those two columns is
// loaded once and used for both, so a Utot element is read from shared memory about
// (NMA + 3) / (2 NMA) times per product instead of twice.  Only the target level j is a
// template parameter: the code of one instantiation stays small enough for the
// instruction cache although the warps of a block work on different rows.

// Guard entries (zeros) before and after the half plane in shared memory: the column
// walks below read up to YR_GUARD entries past either end of a row.  Those reads meet a
// CG factor of exactly zero (the factor tables are zero wherever ma1 or ma2 is out of
// range), so they only have to stay inside the array and be finite.
__host__ __device__ constexpr int yr_guard(int J) { return J + 2; }

// Shared memory of k_snap_yrows, in bytes:
//   front: the triple coefficients [nsp][ntp] (beta-dependent, filled per launch) and the CG
//          factors of every triple (yca), at least yr_guard entries of Utot long;
//   Utot:  the half plane of 32 atoms, [u_half][32] double2;
//   back:  the energy slot of every target row, [rows][32] doubles, at least yr_guard long.
// The out-of-range window reads fall into front or back: finite values (the free parts are
// zeroed) that meet CG factors of exactly zero.
struct YrSmem {
  int ntp, front, u, back;
  __host__ __device__ int total() const { return front + u + back; }
};
__host__ __device__ inline YrSmem yr_smem(int J, int nsp, int ntrip, int nyca, int uh, int nrows) {
  YrSmem m;
  m.ntp = ntrip + (ntrip & 1);
  const int guard = yr_guard(J) * YS_ATOMS * 16;
  const int f = (8 * (nsp * m.ntp + nyca) + 15) & ~15;
  m.front = f > guard ? f : guard;
  m.u = uh * YS_ATOMS * 16;
  const int e = nrows * YS_ATOMS * 8;
  m.back = e > guard ? e : guard;
  return m;
}

// One row pair (mb1, mb2) of a triple for the target-row tile ma = ma0 .. ma0+NT-1.  The
// j1 row is walked as a window: element t of column pair m0 is ma1 = d - m0 - 1 + ma0 + t,
// met by (ma = ma0 + t - 1, ma2 = m0) and (ma = ma0 + t, ma2 = m0 + 1).  cp: the triple's
// factors as [m0/2][ma = 0..j][2], rs = j + 1.
//
// Mirrored rows cost no extra instructions.  M1 (the j1 row lies beyond the half plane):
// U(j1, mb1, ma1) = (-1)^(ma1+mb1) conj(v), and with m0 even the sign splits into
// (-1)^(ma0+d+mb1), folded into cb, times (-1)^(i+q) with i = ma - ma0, a compile-time
// constant folded into the FMAs along with the conjugate.  A mirrored j2 row gives
// (-1)^mb2 (into cb) times (-1)^q and a conjugate, folded into the two per-column scales.
template <int NT, bool M1>
__device__ __forceinline__ void yr_pair(const double2* __restrict__ usl, const int* __restrict__ hblk,
                                        const double2* __restrict__ cp, int rs, int ma0, int j1, int j2, int d,
                                        int mb1, int mb2, double cb, double2 (&acc)[NT]) {
  const double2* p1 = usl + (size_t)(hblk[j1] + (M1 ? j1 - mb1 : mb1) * (j1 + 1) + (M1 ? j1 : 0)) * YS_ATOMS;
  const bool m2 = 2 * mb2 > j2;
  const double2* p2 = usl + (size_t)(hblk[j2] + (m2 ? j2 - mb2 : mb2) * (j2 + 1) + (m2 ? j2 : 0)) * YS_ATOMS;
  const int st2 = m2 ? -YS_ATOMS : YS_ATOMS;
  if (M1 && ((ma0 + d + mb1) & 1)) cb = -cb;
  if (m2 && (mb2 & 1)) cb = -cb;
  const double sx0 = cb, sy0 = m2 ? -cb : cb, sx1 = m2 ? -cb : cb, sy1 = cb;
  cp += ma0;
  int m0 = 0;
  for (; m0 < j2; m0 += 2, cp += rs) {  // column pairs (m0, m0 + 1) both in range
    const double2 v0 = p2[0], v1 = p2[st2];
    p2 += 2 * st2;
    double2 r[2];
    r[0] = make_double2(sx0 * v0.x, sy0 * v0.y);
    r[1] = make_double2(sx1 * v1.x, sy1 * v1.y);
    double2 a[NT];
#pragma unroll
    for (int i = 0; i < NT; i++) a[i] = cp[i];
    const int base = d - m0 - 1 + ma0;
    const double2* pb = p1 + (M1 ? -base : base) * YS_ATOMS;
    double2 u[NT + 1];
#pragma unroll
    for (int t = 0; t <= NT; t++) u[t] = pb[(M1 ? -t : t) * YS_ATOMS];
    // one sweep per column (q = 1: element i, q = 0: element i + 1), so the two updates of an
    // accumulator are NT terms apart; each term forms the complex product first and adds it
    // with one FMA per component
#pragma unroll
    for (int q = 1; q >= 0; q--) {
#pragma unroll
      for (int i = 0; i < NT; i++) {
        const double2 v = u[i + 1 - q];
        const double2 w = r[q];
        double px, py;
        if (M1) {  // conj(v) w
          px = fma(v.x, w.x, v.y * w.y);
          py = fma(v.x, w.y, -(v.y * w.x));
        } else {
          px = fma(v.x, w.x, -(v.y * w.y));
          py = fma(v.x, w.y, v.y * w.x);
        }
        const double c0 = q ? a[i].y : a[i].x;
        const double c = (M1 && ((i + q) & 1)) ? -c0 : c0;
        acc[i].x = fma(c, px, acc[i].x);
        acc[i].y = fma(c, py, acc[i].y);
      }
    }
  }
  if (!(j2 & 1)) {  // even j2: the last column (m0 = j2) alone; its partner j2 + 1 is out of range
    const double2 v0 = p2[0];
    const double2 w = make_double2(sx0 * v0.x, sy0 * v0.y);
    const int base = d - m0 - 1 + ma0;
    const double2* pb = p1 + (M1 ? -base : base) * YS_ATOMS;
#pragma unroll
    for (int i = 0; i < NT; i++) {
      const double2 v = pb[(M1 ? -(i + 1) : (i + 1)) * YS_ATOMS];
      double px, py;
      if (M1) {
        px = fma(v.x, w.x, v.y * w.y);
        py = fma(v.x, w.y, -(v.y * w.x));
      } else {
        px = fma(v.x, w.x, -(v.y * w.y));
        py = fma(v.x, w.y, v.y * w.x);
      }
      const double c0 = cp[i].x;
      const double c = (M1 && (i & 1)) ? -c0 : c0;
      acc[i].x = fma(c, px, acc[i].x);
      acc[i].y = fma(c, py, acc[i].y);
    }
  }
}

// Tile ma0 .. ma0+NT-1 of target row (j, mb): every triple and row pair of the row.
// Writes Y' = w Y of the tile's entries below nma and returns their Re(conj(U) Y').
template <int NT>
__device__ __forceinline__ double yr_tile(const SnapDev& S, const YConst& T, const YRowDev& row, int ma0, int nma,
                                          const double2* __restrict__ usl, const double* __restrict__ yc,
                                          const double2* __restrict__ cas, int64_t n, int64_t atom, bool valid,
                                          double2* __restrict__ yout) {
  double2 acc[NT];
#pragma unroll
  for (int i = 0; i < NT; i++) acc[i] = make_double2(0.0, 0.0);
  const int j = row.j, rs = j + 1;
  const double bn = S.bnorm_flag ? 1.0 / (j + 1) : 1.0;
  for (int t = row.t0; t < row.t1; t++) {
    const YItemDev it = T.items[t];
    const double c = yc[it.trip] * bn;
    const double2* __restrict__ cp = cas + it.ca / 2;
    const int j1 = it.j1, j2 = it.j2, d = it.d;
    for (int ib = 0; ib < it.nb; ib++) {
      const int mb1 = it.mb1min + ib, mb2 = it.mb2max - ib;
      const double cb = c * T.cb[it.cg + ib];  // cg[mb1][mb2] of this row pair
      if (2 * mb1 > j1)
        yr_pair<NT, true>(usl, S.half_block, cp, rs, ma0, j1, j2, d, mb1, mb2, cb, acc);
      else
        yr_pair<NT, false>(usl, S.half_block, cp, rs, ma0, j1, j2, d, mb1, mb2, cb, acc);
    }
  }
  double e = 0.0;
#pragma unroll
  for (int i = 0; i < NT; i++) {
    const int ma = ma0 + i;
    if (ma >= nma) break;
    const double w = (row.mid && ma == nma - 1) ? 0.5 : 1.0;
    const double2 y = make_double2(w * acc[i].x, w * acc[i].y);
    const int h = row.h0 + ma;
    if (valid) yout[(size_t)h * n + atom] = y;
    const double2 u = usl[(size_t)h * YS_ATOMS];
    e += u.x * y.x + u.y * y.y;
  }
  return e;
}

// Tiles of a row of nma entries: at most YR_TILE wide, as even as possible.
#ifndef IPG_YR_TILE
#define IPG_YR_TILE 5  // widths 4, 5, 6 measured 1.80, 1.77, 1.86 ms at 54,000 atoms (eight warps)
#endif
constexpr int YR_TILE = IPG_YR_TILE;

__device__ __forceinline__ double yr_row(const SnapDev& S, const YConst& T, const YRowDev& row,
                                         const double2* __restrict__ usl, const double* __restrict__ yc,
                                         const double2* __restrict__ cas, int64_t n, int64_t atom, bool valid,
                                         double2* __restrict__ yout) {
  const int nma = row.mid ? row.mb + 1 : row.j + 1;
  const int ntile = (nma + YR_TILE - 1) / YR_TILE;
  double e = 0.0;
  int ma0 = 0;
  for (int k = 0; k < ntile; k++) {
    const int w = (nma - ma0 + (ntile - k) - 1) / (ntile - k);  // remaining entries over remaining tiles
    switch (w) {
#define IPG_NT(NT) \
  case NT:         \
    if constexpr (NT <= YR_TILE) e += yr_tile<NT>(S, T, row, ma0, nma, usl, yc, cas, n, atom, valid, yout); \
    break;
      IPG_NT(1) IPG_NT(2) IPG_NT(3) IPG_NT(4) IPG_NT(5) IPG_NT(6)
#undef IPG_NT
      default:
        break;
    }
    ma0 += w;
  }
  return e;
}

// Z output variant (k_snap_yrows<YM_Z>): every item's Z tile goes to zout[jjz][atom]
// (entries of the half plane; the middle row of an even level up to ma = mb), nothing is
// summed across items.  Z carries the 1/(j+1) of bnorm_flag (compute_z.jl:49-56).
template <int NT>
__device__ __forceinline__ void yr_tile_z(const SnapDev& S, const YConst& T, const YRowDev& row, int ma0, int nma,
                                          const double2* __restrict__ usl, const double2* __restrict__ cas, int64_t n,
                                          int64_t atom, bool valid, double2* __restrict__ zout) {
  const int j = row.j, rs = j + 1;
  const double bn = S.bnorm_flag ? 1.0 / (j + 1) : 1.0;
  for (int t = row.t0; t < row.t1; t++) {
    const YItemDev it = T.items[t];
    double2 acc[NT];
#pragma unroll
    for (int i = 0; i < NT; i++) acc[i] = make_double2(0.0, 0.0);
    const double2* __restrict__ cp = cas + it.ca / 2;
    const int j1 = it.j1, j2 = it.j2, d = it.d;
    for (int ib = 0; ib < it.nb; ib++) {
      const int mb1 = it.mb1min + ib, mb2 = it.mb2max - ib;
      const double cb = bn * T.cb[it.cg + ib];
      if (2 * mb1 > j1)
        yr_pair<NT, true>(usl, S.half_block, cp, rs, ma0, j1, j2, d, mb1, mb2, cb, acc);
      else
        yr_pair<NT, false>(usl, S.half_block, cp, rs, ma0, j1, j2, d, mb1, mb2, cb, acc);
    }
    if (valid) {
      const int64_t z0 = it.jjz + row.mb * (j + 1) + ma0;
#pragma unroll
      for (int i = 0; i < NT; i++)
        if (ma0 + i < nma) zout[(size_t)(z0 + i) * n + atom] = acc[i];
    }
  }
}

__device__ __forceinline__ void yr_row_z(const SnapDev& S, const YConst& T, const YRowDev& row,
                                         const double2* __restrict__ usl, const double2* __restrict__ cas, int64_t n,
                                         int64_t atom, bool valid, double2* __restrict__ zout) {
  const int nma = row.mid ? row.mb + 1 : row.j + 1;
  const int ntile = (nma + YR_TILE - 1) / YR_TILE;
  int ma0 = 0;
  for (int k = 0; k < ntile; k++) {
    const int w = (nma - ma0 + (ntile - k) - 1) / (ntile - k);
    switch (w) {
#define IPG_NT(NT) \
  case NT:         \
    if constexpr (NT <= YR_TILE) yr_tile_z<NT>(S, T, row, ma0, nma, usl, cas, n, atom, valid, zout); \
    break;
      IPG_NT(1) IPG_NT(2) IPG_NT(3) IPG_NT(4) IPG_NT(5) IPG_NT(6)
#undef IPG_NT
      default:
        break;
    }
    ma0 += w;
  }
}

// Y and Z at once (k_snap_yrows<YM_YZ>): each item's Z tile is formed with unit coefficients,
// written to zout[jjz][atom] as by yr_tile_z, and added into the row's Y with the item's
// coefficient, so a later beta pullback of the same positions reads Z instead of recomputing
// it.  Y' and the energy are as from yr_tile.
template <int NT>
__device__ __forceinline__ double yr_tile_yz(const SnapDev& S, const YConst& T, const YRowDev& row, int ma0, int nma,
                                             const double2* __restrict__ usl, const double* __restrict__ yc,
                                             const double2* __restrict__ cas, int64_t n, int64_t atom, bool valid,
                                             double2* __restrict__ yout, double2* __restrict__ zout) {
  double2 acc[NT];
#pragma unroll
  for (int i = 0; i < NT; i++) acc[i] = make_double2(0.0, 0.0);
  const int j = row.j, rs = j + 1;
  const double bn = S.bnorm_flag ? 1.0 / (j + 1) : 1.0;
  for (int t = row.t0; t < row.t1; t++) {
    const YItemDev it = T.items[t];
    const double c = yc[it.trip];
    const double2* __restrict__ cp = cas + it.ca / 2;
    const int j1 = it.j1, j2 = it.j2, d = it.d;
    double2 z[NT];
#pragma unroll
    for (int i = 0; i < NT; i++) z[i] = make_double2(0.0, 0.0);
    for (int ib = 0; ib < it.nb; ib++) {
      const int mb1 = it.mb1min + ib, mb2 = it.mb2max - ib;
      const double cb = bn * T.cb[it.cg + ib];
      if (2 * mb1 > j1)
        yr_pair<NT, true>(usl, S.half_block, cp, rs, ma0, j1, j2, d, mb1, mb2, cb, z);
      else
        yr_pair<NT, false>(usl, S.half_block, cp, rs, ma0, j1, j2, d, mb1, mb2, cb, z);
    }
    const int64_t z0 = it.jjz + row.mb * (j + 1) + ma0;
#pragma unroll
    for (int i = 0; i < NT; i++) {
      if (valid && ma0 + i < nma) zout[(size_t)(z0 + i) * n + atom] = z[i];
      acc[i].x = fma(c, z[i].x, acc[i].x);
      acc[i].y = fma(c, z[i].y, acc[i].y);
    }
  }
  double e = 0.0;
#pragma unroll
  for (int i = 0; i < NT; i++) {
    const int ma = ma0 + i;
    if (ma >= nma) break;
    const double w = (row.mid && ma == nma - 1) ? 0.5 : 1.0;
    const double2 y = make_double2(w * acc[i].x, w * acc[i].y);
    const int h = row.h0 + ma;
    if (valid) yout[(size_t)h * n + atom] = y;
    const double2 u = usl[(size_t)h * YS_ATOMS];
    e += u.x * y.x + u.y * y.y;
  }
  return e;
}

__device__ __forceinline__ double yr_row_yz(const SnapDev& S, const YConst& T, const YRowDev& row,
                                            const double2* __restrict__ usl, const double* __restrict__ yc,
                                            const double2* __restrict__ cas, int64_t n, int64_t atom, bool valid,
                                            double2* __restrict__ yout, double2* __restrict__ zout) {
  const int nma = row.mid ? row.mb + 1 : row.j + 1;
  const int ntile = (nma + YR_TILE - 1) / YR_TILE;
  double e = 0.0;
  int ma0 = 0;
  for (int k = 0; k < ntile; k++) {
    const int w = (nma - ma0 + (ntile - k) - 1) / (ntile - k);
    switch (w) {
#define IPG_NT(NT) \
  case NT:         \
    if constexpr (NT <= YR_TILE) e += yr_tile_yz<NT>(S, T, row, ma0, nma, usl, yc, cas, n, atom, valid, yout, zout); \
    break;
      IPG_NT(1) IPG_NT(2) IPG_NT(3) IPG_NT(4) IPG_NT(5) IPG_NT(6)
#undef IPG_NT
      default:
        break;
    }
    ma0 += w;
  }
  return e;
}

// YM: YM_Y writes Y' (yout [u_half][n]) and E_i; YM_Z writes Z (yout [idxz_max][n], nothing
// summed across items); YM_YZ writes both (Z to zout).
// NW: warps per block (the Utot tile of 32 atoms is shared by all of them; two blocks per SM).
constexpr int YM_Y = 0, YM_Z = 1, YM_YZ = 2;
template <int YM, int NW = YS_WARPS>
__global__ void __launch_bounds__(NW * 32, 2) k_snap_yrows(const __grid_constant__ SnapDev S, const __grid_constant__ YConst T, int64_t n,
                                                                 const int32_t* __restrict__ species,
                                                                 const double2* __restrict__ utot,
                                                                 double2* __restrict__ yout, double* __restrict__ Ei,
                                                                 double2* __restrict__ zout) {
  constexpr bool ZOUT = YM == YM_Z;
  extern __shared__ __align__(16) unsigned char ysh[];  // layout: yr_smem
  __shared__ int next_row;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int U = S.idxu_max, UH = S.u_half;
  const YrSmem M = yr_smem(S.J, S.nsp, S.n_ytrip, S.n_yca, UH, S.n_yrows);
  double* ycs = reinterpret_cast<double*>(ysh);  // [nsp][ntp] Y coefficient of each triple
  double* cad = ycs + S.nsp * M.ntp;             // CG factors of every triple
  const double2* cas = reinterpret_cast<const double2*>(cad);
  double2* us = reinterpret_cast<double2*>(ysh + M.front);
  double* erow = reinterpret_cast<double*>(ysh + M.front + M.u);  // [rows][32]
  for (int idx = threadIdx.x; idx < S.nsp * M.ntp; idx += blockDim.x) {
    const int sp = idx / M.ntp, t = idx - sp * M.ntp;
    ycs[idx] = t < S.n_ytrip ? S.ycoef[(size_t)sp * S.idxz_max + S.ytrip_jjz[t]] : 0.0;
  }
  for (int idx = threadIdx.x; idx < S.n_yca; idx += blockDim.x) cad[idx] = S.yca[idx];
  {
    double* gap = cad + S.n_yca;
    const int ngap = (M.front - 8 * (S.nsp * M.ntp + S.n_yca)) / 8;
    for (int idx = threadIdx.x; idx < ngap; idx += blockDim.x) gap[idx] = 0.0;
    for (int idx = threadIdx.x; idx < M.back / 8; idx += blockDim.x) erow[idx] = 0.0;
  }
  for (int64_t a0 = (int64_t)blockIdx.x * YS_ATOMS; a0 < n; a0 += (int64_t)gridDim.x * YS_ATOMS) {
    const int na_blk = (int)((n - a0) < YS_ATOMS ? (n - a0) : YS_ATOMS);
    for (int idx = threadIdx.x; idx < UH * YS_ATOMS; idx += blockDim.x) {
      const int q = idx / YS_ATOMS, l = idx - q * YS_ATOMS;
      us[idx] = l < na_blk ? utot[(size_t)(a0 + l) * U + S.u_of_h[q]] : make_double2(0.0, 0.0);
    }
    if (threadIdx.x == 0) next_row = 0;
    __syncthreads();
    const int64_t atom = a0 + lane;
    const bool valid = lane < na_blk;
    const int si = valid ? clamp_sp(species[atom], S.nsp) : 0;
    const double* yc = ycs + si * M.ntp;
    const double2* usl = us + lane;
    // rows are handed out longest first to whichever warp is free; a row's result does
    // not depend on the warp that computes it, and the energy is summed in row order
    for (;;) {
      int r = 0;
      if (lane == 0) r = atomicAdd(&next_row, 1);
      r = __shfl_sync(0xffffffffu, r, 0);
      if (r >= T.nrows) break;
      const YRowDev row = T.rows[r];
      if (ZOUT)
        yr_row_z(S, T, row, usl, cas, n, atom, valid, yout);  // yout: Z [idxz_max][n]
      else if (YM == YM_YZ)
        erow[r * YS_ATOMS + lane] = yr_row_yz(S, T, row, usl, yc, cas, n, atom, valid, yout, zout);
      else
        erow[r * YS_ATOMS + lane] = yr_row(S, T, row, usl, yc, cas, n, atom, valid, yout);
    }
    __syncthreads();
    if (!ZOUT && warp == 0 && valid) {
      double t = 0.0;
      for (int r = 0; r < T.nrows; r++) t += erow[r * YS_ATOMS + lane];
      Ei[atom] = (2.0 / 3.0) * t + S.ebias[si];
    }
    __syncthreads();
  }
}

// ---- beta pullback from the register chains (twojmax <= YR_MAX_J) -------------------------
// The cotangent g of the forces pulls back to
//   gbeta[s][b] = sum over atoms i of species s of
//                 2 sum_t fac_t sum_half w Re(conj(V_i) Z_i(t)) + gE B_i[b],
//   V_i = sum over neighbors j of (g_i - g_j) . dU_ij/dr_ij      (half plane of every level),
// the terms t, levels and factors of each component being those of dB/dr (compute_b.jl:
// 207-400).  V comes from k_snap_vsum (every chain of a neighbor per lane), Z from
// k_snap_yrows<YM_Z>, and k_snap_gbeta contracts them with the atoms in lanes.

// V of atoms a0 .. a0+nc-1 as V[h][nc]: one warp per atom, lanes over neighbors (32 at a
// time), v_h = A u_h + sum_k B_k du_k,h with A = dsfac gv.uhat, B_k = sfac gv_k, gv = g_i - g_j;
// the sums over lanes go through the staging buffer in fixed order.
constexpr int VS_WARPS = 4;
template <int J>
__global__ void __launch_bounds__(VS_WARPS * 32) k_snap_vsum(const __grid_constant__ SnapDev S, int64_t a0, int64_t nc,
                                                             const int64_t* __restrict__ off,
                                                             const int32_t* __restrict__ nbr,
                                                             const double* __restrict__ rij,
                                                             const int32_t* __restrict__ species,
                                                             const double* __restrict__ g, double2* __restrict__ V) {
  extern __shared__ double2 vsh[];  // saved start rows [4 (J+1)][VS_WARPS 32], then [VS_WARPS][UT_SLOTS 33]
  __shared__ int dst[VS_WARPS][snapchain::UT_SLOTS];
  constexpr int NT = VS_WARPS * 32;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t li = (int64_t)blockIdx.x * VS_WARPS + w;
  if (li >= nc) return;  // warp-uniform; the kernel synchronises only within a warp
  const int64_t i = a0 + li;
  const int si = clamp_sp(species[i], S.nsp);
  const int64_t beg = off[i], end = off[i + 1];
  const double gi0 = g[3 * i], gi1 = g[3 * i + 1], gi2 = g[3 * i + 2];
  snapchain::UtStage st;
  st.buf = vsh + 4 * (J + 1) * NT + w * snapchain::UT_SLOTS * 33;
  st.dst = dst[w];
  st.ut = reinterpret_cast<double*>(V + li);
  st.stride = nc;
  st.lane = lane;
  st.nslot = 0;
  st.wself = 0.0;
  for (int64_t p0 = beg; p0 < (end > beg ? end : beg + 1); p0 += 32) {
    const int64_t p = p0 + lane;
    snapchain::Geom G;  // idle lanes: the identity rotation with zero weights
    G.a = make_double2(1.0, 0.0);
    G.b = make_double2(0.0, 0.0);
    G.sfac = 0.0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      G.da[k] = make_double2(0.0, 0.0);
      G.db[k] = make_double2(0.0, 0.0);
      G.dsu[k] = 0.0;
    }
    double A = 0.0, Bk[3] = {0.0, 0.0, 0.0};
    if (p < end) {
      const int32_t jn = nbr[p];
      const int sj = clamp_sp(species[jn], S.nsp);
      const double rcut = (S.radii[si] + S.radii[sj]) * S.rcutfac;
      PairGeom PG;
      geom_du(S, rij[3 * p], rij[3 * p + 1], rij[3 * p + 2], rcut, S.weight[sj], PG);
      G.a = PG.a;
      G.b = PG.b;
      G.sfac = PG.sfac;
      const double gv[3] = {gi0 - g[3 * jn], gi1 - g[3 * jn + 1], gi2 - g[3 * jn + 2]};
#pragma unroll
      for (int k = 0; k < 3; k++) {
        G.da[k] = PG.da[k];
        G.db[k] = PG.db[k];
        A += gv[k] * (PG.dsfac * PG.u[k]);
        Bk[k] = PG.sfac * gv[k];
      }
    }
    st.first = p0 == beg;
    snapchain::all_chains_v<J>(G, A, Bk, st, vsh, NT, threadIdx.x);
  }
}

// V from U alone (snapchain::all_chains_vlie: the generator identity of k_snap_pair_lie
// applied to the derivative chains of k_snap_vsum).
template <int J>
__global__ void __launch_bounds__(VS_WARPS * 32) k_snap_vlie(const __grid_constant__ SnapDev S, int64_t a0, int64_t nc,
                                                             const int64_t* __restrict__ off,
                                                             const int32_t* __restrict__ nbr,
                                                             const double* __restrict__ rij,
                                                             const int32_t* __restrict__ species,
                                                             const double* __restrict__ g, double2* __restrict__ V) {
  extern __shared__ double2 vsh[];  // [VS_WARPS][UT_SLOTS 33]
  __shared__ int dst[VS_WARPS][snapchain::UT_SLOTS];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t li = (int64_t)blockIdx.x * VS_WARPS + w;
  if (li >= nc) return;  // warp-uniform; the kernel synchronises only within a warp
  const int64_t i = a0 + li;
  const int si = clamp_sp(species[i], S.nsp);
  const int64_t beg = off[i], end = off[i + 1];
  const double gi0 = g[3 * i], gi1 = g[3 * i + 1], gi2 = g[3 * i + 2];
  snapchain::UtStage st;
  st.buf = vsh + w * snapchain::UT_SLOTS * 33;
  st.dst = dst[w];
  st.ut = reinterpret_cast<double*>(V + li);
  st.stride = nc;
  st.lane = lane;
  st.nslot = 0;
  st.wself = 0.0;
  for (int64_t p0 = beg; p0 < (end > beg ? end : beg + 1); p0 += 32) {
    const int64_t p = p0 + lane;
    double2 a = make_double2(1.0, 0.0), b = make_double2(0.0, 0.0);  // idle lanes: zero weights
    double A = 0.0, gm[3] = {0.0, 0.0, 0.0};
    if (p < end) {
      const int32_t jn = nbr[p];
      const int sj = clamp_sp(species[jn], S.nsp);
      const double rcut = (S.radii[si] + S.radii[sj]) * S.rcutfac;
      PairGeom PG;
      geom_du(S, rij[3 * p], rij[3 * p + 1], rij[3 * p + 2], rcut, S.weight[sj], PG);
      a = PG.a;
      b = PG.b;
      const double gv[3] = {gi0 - g[3 * jn], gi1 - g[3 * jn + 1], gi2 - g[3 * jn + 2]};
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const double2 da = PG.da[k], db = PG.db[k];
        A += gv[k] * (PG.dsfac * PG.u[k]);
        const double Bk = PG.sfac * gv[k];
        gm[0] = fma(Bk, a.y * da.x - a.x * da.y + b.x * db.y - b.y * db.x, gm[0]);  // Im(a conj(da) + conj(b) db)
        gm[1] = fma(Bk, b.x * da.x + b.y * da.y - a.x * db.x - a.y * db.y, gm[1]);  // Re(conj(b) da - a conj(db))
        gm[2] = fma(Bk, b.x * da.y - b.y * da.x - a.y * db.x + a.x * db.y, gm[2]);  // Im(conj(b) da - a conj(db))
      }
    }
    st.first = p0 == beg;
    snapchain::all_chains_vlie<J>(a, b, A, gm[0], gm[1], gm[2], st);
  }
}

template <int J>
int launch_vsum_j(ipg_ctx* ctx, const SnapDev& S, int64_t a0, int64_t nc, const int64_t* off, const int32_t* nbr,
                  const double* rij, const int32_t* species, const double* g, double2* V, bool tangent) {
  if (!tangent) {
    const size_t sl = (size_t)VS_WARPS * snapchain::UT_SLOTS * 33 * sizeof(double2);
    if (sl > 48 * 1024)
      CUDA_RET(ctx, cudaFuncSetAttribute(k_snap_vlie<J>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sl));
    IPG_TIMED_LAUNCH(ctx, "snap_vsum", k_snap_vlie<J>, nblk(nc, VS_WARPS), VS_WARPS * 32, sl, S, a0, nc, off, nbr,
                     rij, species, g, V);
    return IPG_OK;
  }
  const size_t sm = ((size_t)4 * (J + 1) * VS_WARPS * 32 + (size_t)VS_WARPS * snapchain::UT_SLOTS * 33) * sizeof(double2);
  if (sm > 48 * 1024)
    CUDA_RET(ctx, cudaFuncSetAttribute(k_snap_vsum<J>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  IPG_TIMED_LAUNCH(ctx, "snap_vsum", k_snap_vsum<J>, nblk(nc, VS_WARPS), VS_WARPS * 32, sm, S, a0, nc, off, nbr, rij,
                   species, g, V);
  return IPG_OK;
}

// tangent: the forward tangent chains (k_snap_vsum) instead of the generator identity (k_snap_vlie)
int launch_vsum(ipg_ctx* ctx, const SnapDev& S, int64_t a0, int64_t nc, const int64_t* off, const int32_t* nbr,
                const double* rij, const int32_t* species, const double* g, double2* V, bool tangent) {
  if (nc == 0) return IPG_OK;
  switch (S.J) {
#define IPG_J(JJ) \
  case JJ:        \
    return launch_vsum_j<JJ>(ctx, S, a0, nc, off, nbr, rij, species, g, V, tangent);
    IPG_J(0) IPG_J(1) IPG_J(2) IPG_J(3) IPG_J(4) IPG_J(5) IPG_J(6) IPG_J(7) IPG_J(8)
#undef IPG_J
    default:
      return IPG_ERR_UNSUPPORTED;
  }
}

// sum over the half plane of level l, entries z0.. of Z: w Re(conj(X) Z), w = 1 below the
// middle element of an even level, 1/2 on it (the weights of compute_b.jl:207-400)
__device__ __forceinline__ double half_dot(const double2* __restrict__ xs, int l, int hb,
                                           const double2* __restrict__ Z, int64_t z0, int64_t zs) {
  const int nf = nfull_of(l);
  const double2* __restrict__ x = xs + (size_t)hb * YS_ATOMS;
  const double2* __restrict__ z = Z + z0 * zs;
  double s0 = 0.0, s1 = 0.0;
  for (int e = 0; e < nf; e++) {
    const double2 a = x[(size_t)e * YS_ATOMS], c = z[e * zs];
    s0 = fma(a.x, c.x, s0);
    s1 = fma(a.y, c.y, s1);
  }
  double s = s0 + s1;
  if (!(l & 1)) {
    const int e = (l / 2) * (l + 1) + l / 2;
    const double2 a = x[(size_t)e * YS_ATOMS], c = z[e * zs];
    s += 0.5 * (a.x * c.x + a.y * c.y);
  }
  return s;
}

// Contraction of V (and, with gE != 0, Utot for B) with Z for atoms a0 .. a0+nc-1: 32 atoms
// per tile in lanes, V (Utot) of the tile staged in shared memory as [u_half][32], the warps
// of a block taking components b = warp, warp + GB_WARPS, ...; per species, the lane values
// are warp sums added in tile order to the block's partial gpart[block][nsp][K].
constexpr int GB_WARPS = 16;
__global__ void __launch_bounds__(GB_WARPS * 32) k_snap_gbeta(const __grid_constant__ SnapDev S, int64_t a0,
                                                              int64_t nc, const int32_t* __restrict__ species,
                                                              const double2* __restrict__ Z,
                                                              const double2* __restrict__ V,
                                                              const double2* __restrict__ utot, double gE,
                                                              double* __restrict__ gpart) {
  extern __shared__ __align__(16) unsigned char gsh[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int UH = S.u_half, K = S.K, nsp = S.nsp;
  const bool withB = gE != 0.0;
  double2* vs = reinterpret_cast<double2*>(gsh);  // [UH][32]
  double2* us = vs + (size_t)UH * YS_ATOMS;       // [UH][32] when withB
  double* gacc = reinterpret_cast<double*>(us + (withB ? (size_t)UH * YS_ATOMS : 0));  // [nsp][K]
  for (int q = threadIdx.x; q < nsp * K; q += blockDim.x) gacc[q] = 0.0;
  const int64_t ntile = (nc + YS_ATOMS - 1) / YS_ATOMS;
  for (int64_t t = blockIdx.x; t < ntile; t += gridDim.x) {
    const int64_t l0 = t * YS_ATOMS;
    const int na = (int)((nc - l0) < YS_ATOMS ? (nc - l0) : YS_ATOMS);
    __syncthreads();  // the previous tile's reads of vs / us are done
    for (int idx = threadIdx.x; idx < UH * YS_ATOMS; idx += blockDim.x) {
      const int q = idx / YS_ATOMS, l = idx - q * YS_ATOMS;
      vs[idx] = l < na ? V[(size_t)q * nc + l0 + l] : make_double2(0.0, 0.0);
      if (withB)
        us[idx] = l < na ? utot[(size_t)(a0 + l0 + l) * S.idxu_max + S.u_of_h[q]] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    const bool valid = lane < na;
    const int64_t la = l0 + (valid ? lane : 0);  // idle lanes read atom l0's Z and drop it
    const int si = valid ? clamp_sp(species[a0 + la], S.nsp) : -1;
    const double2* vl = vs + lane;
    const double2* ul = us + lane;
    const double2* Zl = Z + la;
    for (int b = warp; b < K; b += GB_WARPS) {
      const DBDev d = S.db[b];
      double tot = 0.0;
#pragma unroll
      for (int term = 0; term < 3; term++) {
        const int l = d.l[term];
        tot += d.fac[term] * half_dot(vl, l, S.half_block[l], Zl, d.z0[term], nc);
      }
      double val = 2.0 * tot;
      if (withB) {
        const int l = d.l[0];
        const double B = 2.0 * half_dot(ul, l, S.half_block[l], Zl, d.z0[0], nc) - (S.bzero_flag ? S.bzero[l] : 0.0);
        val += gE * B;
      }
      for (int sp = 0; sp < nsp; sp++) {
        const double x = warp_sum(si == sp ? val : 0.0);
        if (lane == 0) gacc[sp * K + b] += x;
      }
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nsp * K; q += blockDim.x) gpart[(size_t)blockIdx.x * nsp * K + q] = gacc[q];
}

// Bispectrum components from Z (k_snap_yrows<YM_Z>) and Utot for atoms a0 .. a0+nc-1
// (compute_b.jl:17-94): B_b = 2 sum_half w Re(conj(U_j) Z(j1,j2,j)) - bzero_j, 32 atoms per
// tile in lanes, the warps over components; Ei = beta[s_i] . B_i (the bzero shift inside B).
// B [n][K] (optional) and Ei [n] are indexed by the global atom.
__global__ void __launch_bounds__(GB_WARPS * 32) k_snap_bdesc(const __grid_constant__ SnapDev S, int64_t a0,
                                                              int64_t nc, const int32_t* __restrict__ species,
                                                              const double2* __restrict__ Z,
                                                              const double2* __restrict__ utot, double* __restrict__ B,
                                                              double* __restrict__ Ei) {
  extern __shared__ __align__(16) unsigned char bsh[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int UH = S.u_half, K = S.K;
  double2* us = reinterpret_cast<double2*>(bsh);                      // [UH][32]
  double* bs = reinterpret_cast<double*>(us + (size_t)UH * YS_ATOMS);  // [K][32]
  const int64_t ntile = (nc + YS_ATOMS - 1) / YS_ATOMS;
  for (int64_t t = blockIdx.x; t < ntile; t += gridDim.x) {
    const int64_t l0 = t * YS_ATOMS;
    const int na = (int)((nc - l0) < YS_ATOMS ? (nc - l0) : YS_ATOMS);
    __syncthreads();
    for (int idx = threadIdx.x; idx < UH * YS_ATOMS; idx += blockDim.x) {
      const int q = idx / YS_ATOMS, l = idx - q * YS_ATOMS;
      us[idx] = l < na ? utot[(size_t)(a0 + l0 + l) * S.idxu_max + S.u_of_h[q]] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    const bool valid = lane < na;
    const int64_t la = l0 + (valid ? lane : 0);
    for (int b = warp; b < K; b += GB_WARPS) {
      const DBDev d = S.db[b];
      const int l = d.l[0];
      const double v = 2.0 * half_dot(us + lane, l, S.half_block[l], Z + la, d.z0[0], nc) -
                       (S.bzero_flag ? S.bzero[l] : 0.0);
      bs[b * YS_ATOMS + lane] = v;
      if (B && valid) B[(size_t)(a0 + la) * K + b] = v;
    }
    __syncthreads();
    if (warp == 0 && valid) {
      const int si = clamp_sp(species[a0 + la], S.nsp);
      const double* bt = S.beta + (size_t)si * K;
      double e = 0.0;
      for (int b = 0; b < K; b++) e = fma(bt[b], bs[b * YS_ATOMS + lane], e);
      Ei[a0 + la] = e;
    }
  }
}

// ---- plain dB/dr path from the register chains (twojmax <= YR_MAX_J) ----------------------
// dB_i/dr_ij [b][k] = 2 sum_t fac_t sum_half w Re(conj(dU_ij,k) Z_i(t)) (compute_dbidrj.jl;
// compute_b.jl:207-400).  Every Z triple z belongs to one component jjb(z) with one
// multiplier m(z) (its coincidence count and, unnormalised, (j1+1)/(j+1)), the same pair the
// Y coefficients use, so dB[b][k] = 2 sum_{z: jjb(z) = b} m(z) sum_half w Re(conj(dU_k) Z_z).
// k_snap_dbfused computes each pair's dU row by row on the register chains and contracts the
// rows with the owner's Z, the Z triples of a level unrolled at compile time (their tables
// below are constexpr restatements of the host's idxz / idxb / y_jjb / y_mult loops).
namespace plaintab {
constexpr int zrow_count(int j) { return (j / 2 + 1) * (j + 1); }
constexpr int imin(int a, int b) { return a < b ? a : b; }
constexpr int idxb_of(int J, int a, int b, int c) {
  int k = 0;
  for (int j1 = 0; j1 <= J; j1++)
    for (int j2 = 0; j2 <= j1; j2++)
      for (int j = j1 - j2; j <= imin(J, j1 + j2); j += 2)
        if (j >= j1) {
          if (j1 == a && j2 == b && j == c) return k;
          k++;
        }
  return -1;
}
constexpr int nb_of(int J) {
  int k = 0;
  for (int j1 = 0; j1 <= J; j1++)
    for (int j2 = 0; j2 <= j1; j2++)
      for (int j = j1 - j2; j <= imin(J, j1 + j2); j += 2)
        if (j >= j1) k++;
  return k;
}
constexpr int LMAX = 64;
struct Level {  // the Z triples (j1, j2, L) of level L
  int n = 0;
  int z0[LMAX] = {};   // first Z entry
  int jjb[LMAX] = {};  // component
  double m[LMAX] = {}, mn[LMAX] = {};  // multiplier without / with bnorm_flag
};
// Group g of G: the triples whose component b has b % G == g, with jjb = b / G.
constexpr Level level_of(int J, int L, int G = 1, int g = 0) {
  Level T;
  int z = 0;
  for (int j1 = 0; j1 <= J; j1++)
    for (int j2 = 0; j2 <= j1; j2++)
      for (int j = j1 - j2; j <= imin(J, j1 + j2); j += 2) {
        if (j == L && T.n < LMAX) {
          int jjb = 0;
          double mult = 1.0;
          if (j >= j1) {
            jjb = idxb_of(J, j1, j2, j);
            mult = (j1 == j) ? ((j2 == j) ? 3.0 : 2.0) : 1.0;
          } else if (j >= j2) {
            jjb = idxb_of(J, j, j2, j1);
            mult = (j2 == j) ? 2.0 : 1.0;
          } else {
            jjb = idxb_of(J, j2, j, j1);
          }
          if (jjb % G != g) {
            z += zrow_count(j);
            continue;
          }
          T.z0[T.n] = z;
          T.jjb[T.n] = jjb / G;
          T.mn[T.n] = mult;
          T.m[T.n] = (j1 > j) ? mult * (j1 + 1.0) / (j + 1.0) : mult;
          T.n++;
        }
        z += zrow_count(j);
      }
  return T;
}
}  // namespace plaintab

// Plain dB/dr, one block per owner atom, warp-specialised: warp 0 (the producer) runs every
// chain of up to 32 of the owner's pairs, one pair per lane, and hands each half-plane row of
// dU/dr to warps 1..3 (the consumers, one per component k) through three row buffers in
// shared memory; each consumer lane contracts the rows of its pair with the owner's
// Z (staged in shared memory) into the 55 accumulators of dB[b][k].  dU never leaves the SM.
// Hand-off by named barriers (ids 1..3: row buffer b full; 4..6: row buffer b free), DBF_T
// threads each: the producer arrives on "full" and waits on "free", the consumers the
// reverse; both sides walk the same row sequence, so every barrier generation completes.
constexpr int DBF_T = 128;

template <int ID>
__device__ __forceinline__ void nbar_sync() {
  asm volatile("bar.sync %0, %1;" ::"n"(ID), "n"(DBF_T) : "memory");
}
template <int ID>
__device__ __forceinline__ void nbar_arrive() {
  asm volatile("bar.arrive %0, %1;" ::"n"(ID), "n"(DBF_T) : "memory");
}
// DBF_NBUF row buffers; buffer b: "full" is barrier 1 + b, "free" is barrier 4 + b (immediate ids)
constexpr int DBF_NBUF = 3;
__device__ __forceinline__ void row_full_arrive(int b) {
  b == 0 ? nbar_arrive<1>() : (b == 1 ? nbar_arrive<2>() : nbar_arrive<3>());
}
__device__ __forceinline__ void row_full_wait(int b) { b == 0 ? nbar_sync<1>() : (b == 1 ? nbar_sync<2>() : nbar_sync<3>()); }
__device__ __forceinline__ void row_free_arrive(int b) {
  b == 0 ? nbar_arrive<4>() : (b == 1 ? nbar_arrive<5>() : nbar_arrive<6>());
}
__device__ __forceinline__ void row_free_wait(int b) { b == 0 ? nbar_sync<4>() : (b == 1 ? nbar_sync<5>() : nbar_sync<6>()); }

template <int J>
struct DbRowEmit {  // producer side: dU_k[ma] of this lane's pair into row buffer r % DBF_NBUF
  const snapchain::Geom& G;
  double2* rows;  // [2][3][J+1][32]
  int lane, r;
  template <int j>
  __device__ __forceinline__ void row(const snapchain::Chain<J>& s, int mb) {
    const int b = r % DBF_NBUF;
    row_free_wait(b);  // the consumers are done with row r - DBF_NBUF
    double2* rb = rows + b * 3 * (J + 1) * 32 + lane;
    const int last = (2 * mb == j) ? mb : j;
#pragma unroll
    for (int ma = 0; ma <= j; ma++) {
      if (ma > last) break;
#pragma unroll
      for (int k = 0; k < 3; k++)
        rb[(k * (J + 1) + ma) * 32] = make_double2(fma(G.dsu[k], s.u[ma].x, G.sfac * s.d[k][ma].x),
                                                   fma(G.dsu[k], s.u[ma].y, G.sfac * s.d[k][ma].y));
    }
    row_full_arrive(b);
    r++;
  }
};

// consumer side: row mb of level L.  The row's entries ma run in a loop; the level's Z triples
// are unrolled inside it (one Z load and two FMAs each), so the code per level stays small.
template <int J, int L, int Q, int NQ>
__device__ __forceinline__ void dbf_dot(double (&c)[NQ], double2 d, const double2* __restrict__ zr) {
  if constexpr (Q < NQ) {
    constexpr int z0 = plaintab::level_of(J, L).z0[Q];
    const double2 z = zr[z0];
    c[Q] = fma(d.x, z.x, fma(d.y, z.y, c[Q]));
    dbf_dot<J, L, Q + 1, NQ>(c, d, zr);
  }
}

template <int J, int L, int Q, int NQ, int NB>
__device__ __forceinline__ void dbf_add(double (&acc)[NB], const double (&c)[NQ], bool bnorm) {
  if constexpr (Q < NQ) {
    constexpr plaintab::Level T = plaintab::level_of(J, L);
    constexpr int b = T.jjb[Q];
    constexpr double m = T.m[Q], mn = T.mn[Q];
    acc[b] = fma(bnorm ? mn : m, c[Q], acc[b]);
    dbf_add<J, L, Q + 1, NQ, NB>(acc, c, bnorm);
  }
}

template <int J, int L, int NB>
__device__ __forceinline__ void dbf_row(double (&acc)[NB], int mb, const double2* __restrict__ rb,
                                        const double2* __restrict__ zo, bool bnorm) {
  if constexpr (L <= J) {
    constexpr int NQ = plaintab::level_of(J, L).n;
    const int last = (2 * mb == L) ? mb : L;
    const double2* zr = zo + mb * (L + 1);
    double c[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) c[q] = 0.0;
#pragma unroll 1
    for (int ma = 0; ma <= last; ma++) {
      double2 d = rb[ma * 32];
      if (2 * mb == L && ma == mb) {  // the middle element of an even level: weight 1/2
        d.x *= 0.5;
        d.y *= 0.5;
      }
      dbf_dot<J, L, 0, NQ>(c, d, zr + ma);
    }
    dbf_add<J, L, 0, NQ, NB>(acc, c, bnorm);
  }
}

template <int J, int NB>
__device__ __forceinline__ void dbf_consume(double (&acc)[NB], int j, int mb, const double2* __restrict__ rb,
                                            const double2* __restrict__ zo, bool bnorm) {
  switch (j) {
#define IPG_L(LL) \
  case LL:        \
    dbf_row<J, LL, NB>(acc, mb, rb, zo, bnorm); \
    break;
    IPG_L(0) IPG_L(1) IPG_L(2) IPG_L(3) IPG_L(4) IPG_L(5) IPG_L(6) IPG_L(7) IPG_L(8)
#undef IPG_L
    default:
      break;
  }
}

// dbl[p][b][k] for the pairs of owners b0 .. b1-1; their Z in the chunk of atoms a0.. (stride zs)
template <int J>
__global__ void __launch_bounds__(DBF_T, 2) k_snap_dbfused(const __grid_constant__ SnapDev S, int64_t b0,
                                                           const int64_t* __restrict__ off,
                                                           const int32_t* __restrict__ nbr,
                                                           const double* __restrict__ rij,
                                                           const int32_t* __restrict__ species, int64_t a0,
                                                           int64_t zs, const double2* __restrict__ Z,
                                                           double* __restrict__ dbl) {
  static_assert(J <= YR_MAX_J, "fused plain kernel covers twojmax <= 8");
  constexpr int NB = plaintab::nb_of(J);
  extern __shared__ __align__(16) unsigned char fsm[];
  double2* zo = reinterpret_cast<double2*>(fsm);                 // [idxz_max] the owner's Z
  double2* rows = zo + ((S.idxz_max + 1) & ~1);                  // [DBF_NBUF][3][J+1][32]
  double2* save = rows + DBF_NBUF * 3 * (J + 1) * 32;            // [4 (J+1)][32] producer start rows
  const int64_t o = b0 + blockIdx.x;
  for (int z = threadIdx.x; z < S.idxz_max; z += DBF_T) zo[z] = Z[(size_t)z * zs + (o - a0)];
  __syncthreads();
  const int64_t pb = off[o], pe = off[o + 1];
  const int npass = (int)((pe - pb + 31) / 32);  // block-uniform
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (npass == 0) return;
  if (warp == 0) {
    const int si = clamp_sp(species[o], S.nsp);
    int r = 0;  // rows handed over so far
    for (int pass = 0; pass < npass; pass++) {
      const int64_t p = pb + pass * 32 + lane;
      snapchain::Geom G;  // idle lanes: the identity rotation with zero weights
      G.a = make_double2(1.0, 0.0);
      G.b = make_double2(0.0, 0.0);
      G.sfac = 0.0;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        G.da[k] = make_double2(0.0, 0.0);
        G.db[k] = make_double2(0.0, 0.0);
        G.dsu[k] = 0.0;
      }
      if (p < pe) {
        const int sj = clamp_sp(species[nbr[p]], S.nsp);
        const double rcut = (S.radii[si] + S.radii[sj]) * S.rcutfac;
        PairGeom PG;
        geom_du(S, rij[3 * p], rij[3 * p + 1], rij[3 * p + 2], rcut, S.weight[sj], PG);
        G.a = PG.a;
        G.b = PG.b;
        G.sfac = PG.sfac;
#pragma unroll
        for (int k = 0; k < 3; k++) {
          G.da[k] = PG.da[k];
          G.db[k] = PG.db[k];
          G.dsu[k] = PG.dsfac * PG.u[k];
        }
      }
      DbRowEmit<J> e{G, rows, lane, r};
      snapchain::all_chains_rows<J>(G, e, save, 32, lane);
      r = e.r;
    }
#pragma unroll
    for (int t = 0; t < DBF_NBUF; t++) row_free_wait((r + t) % DBF_NBUF);  // the consumers' last arrivals
  } else {
    const int k = warp - 1;
    const bool bnorm = S.bnorm_flag != 0;
#pragma unroll
    for (int b = 0; b < DBF_NBUF; b++) row_free_arrive(b);  // every row buffer starts free
    int r = 0;
    for (int pass = 0; pass < npass; pass++) {
      double acc[NB];
#pragma unroll
      for (int b = 0; b < NB; b++) acc[b] = 0.0;
      for (int mb = -1; mb <= J / 2; mb++) {  // mb = -1: the row (0, 0)
        const int j0 = mb < 0 ? 0 : (mb == 0 ? 1 : 2 * mb), j1 = mb < 0 ? 0 : J;
        for (int j = j0; j <= j1; j++, r++) {
          const int bsel = r % DBF_NBUF;
          row_full_wait(bsel);
          dbf_consume<J, NB>(acc, j, mb < 0 ? 0 : mb, rows + (bsel * 3 + k) * (J + 1) * 32 + lane, zo, bnorm);
          row_free_arrive(bsel);
        }
      }
      const int64_t p = pb + pass * 32 + lane;
      if (p < pe) {
        double* out = dbl + (size_t)p * NB * 3 + k;
#pragma unroll
        for (int b = 0; b < NB; b++) out[3 * b] = 2.0 * acc[b];
      }
    }
  }
}

template <int J>
int plain_fused_j(ipg_ctx* ctx, const SnapDev& S, int64_t b0, int64_t b1, const int64_t* off, const int32_t* nbr,
                  const double* rij, const int32_t* species, int64_t a0, int64_t zs, const double2* Z, double* dbl) {
  if constexpr (J > YR_MAX_J) {
    return IPG_ERR_UNSUPPORTED;
  } else {
    if (plaintab::nb_of(J) != S.K) return ipg_fail(ctx, IPG_ERR_UNSUPPORTED, "plain chain tables disagree");
    const size_t sm =
        ((size_t)((S.idxz_max + 1) & ~1) + DBF_NBUF * 3 * (J + 1) * 32 + 4 * (J + 1) * 32) * sizeof(double2);
    if (sm > 48 * 1024)
      CUDA_RET(ctx, cudaFuncSetAttribute(k_snap_dbfused<J>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    IPG_TIMED_LAUNCH(ctx, "snap_dbfused", k_snap_dbfused<J>, (unsigned)(b1 - b0), DBF_T, sm, S, b0, off, nbr, rij,
                     species, a0, zs, Z, dbl);
    return IPG_OK;
  }
}

int plain_fused(ipg_ctx* ctx, const SnapDev& S, int64_t b0, int64_t b1, const int64_t* off, const int32_t* nbr,
                const double* rij, const int32_t* species, int64_t a0, int64_t zs, const double2* Z, double* dbl) {
  if (b1 <= b0) return IPG_OK;
  switch (S.J) {
#define IPG_J(JJ) \
  case JJ:        \
    return plain_fused_j<JJ>(ctx, S, b0, b1, off, nbr, rij, species, a0, zs, Z, dbl);
    IPG_J(0) IPG_J(1) IPG_J(2) IPG_J(3) IPG_J(4) IPG_J(5) IPG_J(6) IPG_J(7) IPG_J(8)
#undef IPG_J
    default:
      return IPG_ERR_UNSUPPORTED;
  }
}

// Adjoint per-neighbor kernel: one thread per (directed pair, chain MB); see
// ipg_snap_chain.cuh.  Yw is the weighted Y as [h][natoms]; part[p][MB][3] = chain MB's
// share of dE_i/dr_ij.
template <int J, int MB>
__global__ void __launch_bounds__(128) k_snap_pair_adj(const __grid_constant__ SnapDev S, const int64_t* __restrict__ d_np, int64_t natoms,
                                                       const int32_t* __restrict__ owner,
                                                       const int32_t* __restrict__ nbr, const double* __restrict__ rij,
                                                       const int32_t* __restrict__ species,
                                                       const double2* __restrict__ Yw, double* __restrict__ part) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= *d_np) return;  // np: the live count (capacity mode sizes the grid larger)
  const int i = owner[p];
  const int si = clamp_sp(species[i], S.nsp), sj = clamp_sp(species[nbr[p]], S.nsp);
  const double rcut = (S.radii[si] + S.radii[sj]) * S.rcutfac;
  PairGeom PG;
  geom_du(S, rij[3 * p], rij[3 * p + 1], rij[3 * p + 2], rcut, S.weight[sj], PG);
  snapchain::Geom G;
  G.a = PG.a;
  G.b = PG.b;
  G.sfac = PG.sfac;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    G.da[k] = PG.da[k];
    G.db[k] = PG.db[k];
    G.dsu[k] = PG.dsfac * PG.u[k];
  }
  double S0, Sk[3];
  snapchain::chain_adjoint<J, MB>(G, Yw + i, natoms, S0, Sk);
  constexpr int NCH = J / 2 + 1;
  double* out = part + ((size_t)p * NCH + MB) * 3;
#pragma unroll
  for (int k = 0; k < 3; k++) out[k] = 2.0 * (G.dsu[k] * S0 + G.sfac * Sk[k]);
}

// Adjoint per-neighbor kernel, all chains of a pair in one thread (saved start rows in
// shared memory): part[p][0][3] = dE_i/dr_ij.
constexpr int PAIR_ALL_T = 128;
constexpr int PAIR_Y_ATOMS = 8;  // atoms whose Y a block of the all-chains kernel stages
template <int J>
__global__ void __launch_bounds__(PAIR_ALL_T) k_snap_pair_adj_all(const __grid_constant__ SnapDev S,
                                                                  const int64_t* __restrict__ d_np,
                                                                  int64_t natoms, const int32_t* __restrict__ owner,
                                                                  const int32_t* __restrict__ nbr,
                                                                  const double* __restrict__ rij,
                                                                  const int32_t* __restrict__ species,
                                                                  const double2* __restrict__ Yw,
                                                                  double* __restrict__ part, int ystage) {
  extern __shared__ double2 save[];  // [4 (J+1)][PAIR_ALL_T], then the staged Y [u_half][PAIR_Y_ATOMS]
  const int64_t np = *d_np;  // the live count (capacity mode sizes the grid larger)
  const int64_t p0 = (int64_t)blockIdx.x * blockDim.x, p = p0 + threadIdx.x;
  if (p0 >= np) return;  // block-uniform
  // The block's pairs are sorted by owner: stage the weighted Y of their few atoms in shared
  // memory (every Y entry is read once per neighbor), unless they span too many atoms.
  const int first = owner[p0];
  const int nat = owner[(p0 + blockDim.x - 1 < np ? p0 + blockDim.x : np) - 1] - first + 1;
  const bool staged = nat <= ystage;  // ystage: 0 (no staging room) or PAIR_Y_ATOMS
  double2* ysm = save + 4 * (J + 1) * PAIR_ALL_T;
  if (staged) {
    for (int idx = threadIdx.x; idx < S.u_half * nat; idx += blockDim.x) {
      const int h = idx / nat, a = idx - h * nat;
      ysm[h * PAIR_Y_ATOMS + a] = Yw[(size_t)h * natoms + first + a];
    }
  }
  __syncthreads();
  if (p >= np) return;
  const int i = owner[p];
  const int si = clamp_sp(species[i], S.nsp), sj = clamp_sp(species[nbr[p]], S.nsp);
  const double rcut = (S.radii[si] + S.radii[sj]) * S.rcutfac;
  PairGeom PG;
  geom_du(S, rij[3 * p], rij[3 * p + 1], rij[3 * p + 2], rcut, S.weight[sj], PG);
  snapchain::Geom G;
  G.a = PG.a;
  G.b = PG.b;
  G.sfac = PG.sfac;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    G.da[k] = PG.da[k];
    G.db[k] = PG.db[k];
    G.dsu[k] = PG.dsfac * PG.u[k];
  }
  double S0, Sk[3];
  if (staged)
    snapchain::all_chains_adjoint<J>(G, ysm + (i - first), PAIR_Y_ATOMS, S0, Sk, save, PAIR_ALL_T, threadIdx.x);
  else
    snapchain::all_chains_adjoint<J>(G, Yw + i, natoms, S0, Sk, save, PAIR_ALL_T, threadIdx.x);
  double* out = part + (size_t)p * 3;
#pragma unroll
  for (int k = 0; k < 3; k++) out[k] = 2.0 * (G.dsu[k] * S0 + G.sfac * Sk[k]);
}

template <int J>
int launch_pair_all(ipg_ctx* ctx, const SnapDev& S, int64_t np, const int64_t* d_np, int64_t natoms, const int32_t* owner,
                    const int32_t* nbr, const double* rij, const int32_t* species, const double2* Yw, double* part) {
  // stage Y only while two blocks (the register limit) still fit an SM's shared memory
  const size_t base = (size_t)4 * (J + 1) * PAIR_ALL_T * sizeof(double2);
  const size_t with_y = base + (size_t)S.u_half * PAIR_Y_ATOMS * sizeof(double2);
  const int ystage = with_y <= 113 * 1024 ? PAIR_Y_ATOMS : 0;
  const size_t sm = ystage ? with_y : base;
  if (sm > 48 * 1024)
    CUDA_RET(ctx, cudaFuncSetAttribute(k_snap_pair_adj_all<J>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  IPG_TIMED_LAUNCH(ctx, "snap_pair", k_snap_pair_adj_all<J>, nblk(np, PAIR_ALL_T), PAIR_ALL_T, sm, S, d_np, natoms,
                   owner, nbr, rij, species, Yw, part, ystage);
  return IPG_OK;
}

int launch_pair_adj_all(ipg_ctx* ctx, const SnapDev& S, int64_t np, const int64_t* d_np, int64_t natoms, const int32_t* owner,
                        const int32_t* nbr, const double* rij, const int32_t* species, const double2* Yw,
                        double* part) {
  if (np == 0) return IPG_OK;
  switch (S.J) {
#define IPG_J(JJ) \
  case JJ:        \
    return launch_pair_all<JJ>(ctx, S, np, d_np, natoms, owner, nbr, rij, species, Yw, part);
    IPG_J(0) IPG_J(1) IPG_J(2) IPG_J(3) IPG_J(4) IPG_J(5) IPG_J(6) IPG_J(7) IPG_J(8) IPG_J(9) IPG_J(10)
#undef IPG_J
    default:
      return IPG_ERR_UNSUPPORTED;
  }
}

// Adjoint forces of every directed pair from U alone (snapchain::all_chains_lie: the
// derivative of U along r_ij is U times a Lie-algebra generator, so the three tangent chains
// of k_snap_pair_adj_all are not needed).  The block's pairs are sorted by owner; the owners'
// weighted Y and the two generator-shifted copies Y2, Y3 (per atom, from Yw) are staged in
// shared memory for up to PAIR_LIE_ATOMS atoms at a time; a block whose pairs span more
// atoms stages them group by group.
constexpr int PAIR_LIE_T = 128;
constexpr int PAIR_LIE_ATOMS = 8;
__host__ __device__ constexpr size_t pair_lie_smem(int uh) { return (size_t)3 * uh * PAIR_LIE_ATOMS * sizeof(double2); }
template <int J>
__global__ void __launch_bounds__(PAIR_LIE_T) k_snap_pair_lie(const __grid_constant__ SnapDev S,
                                                              const int64_t* __restrict__ d_np, int64_t natoms,
                                                              const int32_t* __restrict__ owner,
                                                              const int32_t* __restrict__ nbr,
                                                              const double* __restrict__ rij,
                                                              const int32_t* __restrict__ species,
                                                              const double2* __restrict__ Yw,
                                                              double* __restrict__ part) {
  extern __shared__ double2 ylie[];  // [3][u_half][PAIR_LIE_ATOMS]: Yw, Y2, Y3 of a group of owners
  const int64_t np = *d_np;          // the live count (capacity mode sizes the grid larger)
  const int64_t p0 = (int64_t)blockIdx.x * blockDim.x, p = p0 + threadIdx.x;
  if (p0 >= np) return;  // block-uniform
  const int first = owner[p0];
  const int lastat = owner[(p0 + blockDim.x < np ? p0 + blockDim.x : np) - 1];
  const int UH = S.u_half;
  const int i = p < np ? owner[p] : -1;
  // the first group's Y' goes to shared memory by asynchronous copies (zero-filled beyond each
  // row's weighted entries, which the Y kernel leaves unset) while the pair geometry is computed
  auto stage = [&](int g0, int nat) {
    for (int idx = threadIdx.x; idx < UH * nat; idx += blockDim.x) {
      const int h = idx / nat, at = idx - h * nat;
      const unsigned dst = (unsigned)__cvta_generic_to_shared(ylie + (size_t)h * PAIR_LIE_ATOMS + at);
      const double2* src = Yw + (size_t)h * natoms + g0 + at;
      const int bytes = (S.h_info[h] >> 16) ? 16 : 0;
      asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  stage(first, lastat - first + 1 < PAIR_LIE_ATOMS ? lastat - first + 1 : PAIR_LIE_ATOMS);
  // per direction k: F_k = c0_k S0 + cT_k . T (the generator coefficients times sfac)
  double2 a = make_double2(1.0, 0.0), b = make_double2(0.0, 0.0);
  double c0[3] = {0.0, 0.0, 0.0}, cT[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
  if (p < np) {
    const int si = clamp_sp(species[i], S.nsp), sj = clamp_sp(species[nbr[p]], S.nsp);
    const double rcut = (S.radii[si] + S.radii[sj]) * S.rcutfac;
    PairGeom PG;
    geom_du(S, rij[3 * p], rij[3 * p + 1], rij[3 * p + 2], rcut, S.weight[sj], PG);
    a = PG.a;
    b = PG.b;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const double2 da = PG.da[k], db = PG.db[k];
      c0[k] = 2.0 * PG.dsfac * PG.u[k];
      const double f = 2.0 * PG.sfac;
      cT[k][0] = f * (a.y * da.x - a.x * da.y + b.x * db.y - b.y * db.x);  // Im(a conj(da) + conj(b) db)
      cT[k][1] = f * (b.x * da.x + b.y * da.y - a.x * db.x - a.y * db.y);  // Re(conj(b) da - a conj(db))
      cT[k][2] = f * (b.x * da.y - b.y * da.x - a.y * db.x + a.x * db.y);  // Im(conj(b) da - a conj(db))
    }
  }
  double S0 = 0.0, T[3] = {0.0, 0.0, 0.0};
  for (int g0 = first; g0 <= lastat; g0 += PAIR_LIE_ATOMS) {  // block-uniform bounds
    const int nat = lastat - g0 + 1 < PAIR_LIE_ATOMS ? lastat - g0 + 1 : PAIR_LIE_ATOMS;
    if (g0 > first) {
      __syncthreads();  // the previous group's readers are done
      stage(g0, nat);
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    // Y2, Y3 from the row neighbours of each entry
    for (int idx = threadIdx.x; idx < UH * nat; idx += blockDim.x) {
      const int h = idx / nat, a = idx - h * nat;
      const int inf = S.h_info[h], m = inf & 255, j = (inf >> 8) & 255;
      const double2 sg = S.h_sgen[h];  // (s_m, s_{m-1}), zero where the neighbour is off the row
      const double2 z = make_double2(0.0, 0.0);
      const double2 wp = m < j ? ylie[(size_t)(h + 1) * PAIR_LIE_ATOMS + a] : z;
      const double2 wm = m >= 1 ? ylie[(size_t)(h - 1) * PAIR_LIE_ATOMS + a] : z;
      const double2 A = make_double2(sg.x * wp.x, sg.x * wp.y), B = make_double2(sg.y * wm.x, sg.y * wm.y);
      ylie[(size_t)(UH + h) * PAIR_LIE_ATOMS + a] = make_double2(A.x - B.x, A.y - B.y);
      ylie[(size_t)(2 * UH + h) * PAIR_LIE_ATOMS + a] = make_double2(A.y + B.y, -(A.x + B.x));
    }
    __syncthreads();
    if (i >= g0 && i < g0 + nat)
      snapchain::all_chains_lie<J>(a, b, ylie + (i - g0), PAIR_LIE_ATOMS, UH, S0, T);
  }
  if (p >= np) return;
  double* out = part + (size_t)p * 3;
#pragma unroll
  for (int k = 0; k < 3; k++) out[k] = c0[k] * S0 + (cT[k][0] * T[0] + cT[k][1] * T[1] + cT[k][2] * T[2]);
}

template <int J>
int launch_pair_lie_t(ipg_ctx* ctx, const SnapDev& S, int64_t np, const int64_t* d_np, int64_t natoms,
                      const int32_t* owner, const int32_t* nbr, const double* rij, const int32_t* species,
                      const double2* Yw, double* part) {
  const size_t sm = pair_lie_smem(S.u_half);
  if (sm > 48 * 1024)
    CUDA_RET(ctx, cudaFuncSetAttribute(k_snap_pair_lie<J>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  IPG_TIMED_LAUNCH(ctx, "snap_pair", k_snap_pair_lie<J>, nblk(np, PAIR_LIE_T), PAIR_LIE_T, sm, S, d_np, natoms, owner,
                   nbr, rij, species, Yw, part);
  return IPG_OK;
}

int launch_pair_lie(ipg_ctx* ctx, const SnapDev& S, int64_t np, const int64_t* d_np, int64_t natoms, const int32_t* owner,
                    const int32_t* nbr, const double* rij, const int32_t* species, const double2* Yw, double* part) {
  if (np == 0) return IPG_OK;
  switch (S.J) {
#define IPG_J(JJ) \
  case JJ:        \
    return launch_pair_lie_t<JJ>(ctx, S, np, d_np, natoms, owner, nbr, rij, species, Yw, part);
    IPG_J(0) IPG_J(1) IPG_J(2) IPG_J(3) IPG_J(4) IPG_J(5) IPG_J(6) IPG_J(7) IPG_J(8) IPG_J(9) IPG_J(10)
#undef IPG_J
    default:
      return IPG_ERR_UNSUPPORTED;
  }
}

// ---- exact Hessian-vector product on the register chains -------------------------------
// The position pullback needs Hv, the tangent of the forces along a displacement v of the
// atoms.  dE_i/dr_ij = 2 sum_h w Re(conj(D_k,h) Y_h), D_k = dsfac uhat_k U + sfac dU/dr_k,
// depends on the pair geometry and on the centre atom's Y.  Its tangent along rdot = v_j - v_i
// has a pair-local part (U, dU and the geometry along rdot: the second-order chain of
// snapchain::all_chains_hvp) and a Y part (Ydot).  Y is a quadratic form in Utot, so
// Ydot = [Y(U + s Udot) - Y(U - s Udot)] / (2s) exactly in exact arithmetic (the terms in s^2
// cancel identically; no truncation term), with s a power of two per atom that gives U and
// s Udot the same magnitude; Udot comes from k_snap_vsum (V with g = v is -Udot).

// Per atom (one warp): s = 2^k with s max|Udot| ~ max|U| over the half plane, and the half
// plane of U -/+ s V into Up / Um (full Utot layout; the Y kernel reads only these entries).
// V holds the half plane up to the middle element of an even level; the entries beyond it are
// the inversion-symmetric mirrors of entries of the same row (compute_ui.jl:105-125).
__global__ void k_hvp_split(const __grid_constant__ SnapDev S, int64_t n, const double2* __restrict__ utot,
                            const double2* __restrict__ V, double2* __restrict__ Up, double2* __restrict__ Um,
                            double* __restrict__ scale) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;  // warp-uniform
  const int U = S.idxu_max, UH = S.u_half;
  auto vdot = [&](int h) -> double2 {  // Udot = -V, mirrored where V is not stored
    int j = 0;
    while (j < S.J && S.half_block[j + 1] <= h) j++;
    const int e = h - S.half_block[j], mb = e / (j + 1), ma = e - mb * (j + 1);
    if (2 * mb == j && ma > mb) {
      const double2 m = V[(size_t)(S.half_block[j] + mb * (j + 1) + (j - ma)) * n + i];
      const double sg = ((ma + mb) & 1) ? -1.0 : 1.0;
      return make_double2(-sg * m.x, sg * m.y);  // -( (-1)^(ma+mb) conj(m) )
    }
    const double2 v = V[(size_t)h * n + i];
    return make_double2(-v.x, -v.y);
  };
  double mu = 0.0, mv = 0.0;
  for (int h = lane; h < UH; h += 32) {
    const double2 u = utot[(size_t)i * U + S.u_of_h[h]], d = vdot(h);
    mu = fmax(mu, fmax(fabs(u.x), fabs(u.y)));
    mv = fmax(mv, fmax(fabs(d.x), fabs(d.y)));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mu = fmax(mu, __shfl_xor_sync(0xffffffffu, mu, o));
    mv = fmax(mv, __shfl_xor_sync(0xffffffffu, mv, o));
  }
  int ex = 0;
  if (mv > 0.0 && mu > 0.0) {  // s = 2^round(log2(mu / mv)), exact to multiply and divide by
    int eu, ev;
    frexp(mu, &eu);
    frexp(mv, &ev);
    ex = eu - ev;
  }
  const double s = ldexp(1.0, ex);
  if (lane == 0) scale[i] = s;
  for (int h = lane; h < UH; h += 32) {
    const size_t e = (size_t)i * U + S.u_of_h[h];
    const double2 u = utot[e], d = vdot(h);
    Up[e] = make_double2(fma(s, d.x, u.x), fma(s, d.y, u.y));
    Um[e] = make_double2(fma(-s, d.x, u.x), fma(-s, d.y, u.y));
  }
}

// Ydot[h][i] = (Yp - Ym) / (2 s_i)
__global__ void k_hvp_ydot(int64_t n, int uh, const double2* __restrict__ Yp, const double2* __restrict__ Ym,
                           const double* __restrict__ scale, double2* __restrict__ Yd) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)uh * n) return;
  const int64_t i = t % n;
  const double f = 0.5 / scale[i];
  const double2 a = Yp[t], b = Ym[t];
  Yd[t] = make_double2((a.x - b.x) * f, (a.y - b.y) * f);
}

// fdot[p][k] = the tangent of dE_i/dr_ij[k] along v (one (pair, k) per thread, k = blockIdx.y):
//   2 (cudot T0 + cu T2 + sfacdot T1 + sfac T3 + cu T4 + sfac T5),  cu = dsfac uhat_k,
// T as in snapchain::all_chains_hvp.  Each block stages Y and Ydot of its pairs' few owner
// atoms in shared memory, as k_snap_pair_adj_all does.
constexpr int HVP_T = 128;
constexpr int HVP_Y_ATOMS = 7;
template <int J>
__global__ void __launch_bounds__(HVP_T) k_snap_pair_hvp(const __grid_constant__ SnapDev S,
                                                         const int64_t* __restrict__ d_np, int64_t natoms,
                                                         const int32_t* __restrict__ owner,
                                                         const int32_t* __restrict__ nbr,
                                                         const double* __restrict__ rij,
                                                         const int32_t* __restrict__ species,
                                                         const double* __restrict__ v,
                                                         const double2* __restrict__ Yw,
                                                         const double2* __restrict__ Yd, double* __restrict__ fdot,
                                                         int ystage) {
  extern __shared__ double2 save[];  // [4 (J+1)][HVP_T], then Y and Ydot [2][u_half][HVP_Y_ATOMS]
  const int64_t np = *d_np;
  const int64_t p0 = (int64_t)blockIdx.x * blockDim.x, p = p0 + threadIdx.x;
  if (p0 >= np) return;  // block-uniform
  const int k = blockIdx.y;
  const int first = owner[p0];
  const int nat = owner[(p0 + blockDim.x - 1 < np ? p0 + blockDim.x : np) - 1] - first + 1;
  const bool staged = nat <= ystage;
  double2* ysm = save + 4 * (J + 1) * HVP_T;
  double2* ydm = ysm + S.u_half * HVP_Y_ATOMS;
  if (staged) {
    for (int idx = threadIdx.x; idx < S.u_half * nat; idx += blockDim.x) {
      const int h = idx / nat, a = idx - h * nat;
      ysm[h * HVP_Y_ATOMS + a] = Yw[(size_t)h * natoms + first + a];
      ydm[h * HVP_Y_ATOMS + a] = Yd[(size_t)h * natoms + first + a];
    }
  }
  __syncthreads();
  if (p >= np) return;
  const int i = owner[p];
  const int32_t jn = nbr[p];
  const int si = clamp_sp(species[i], S.nsp), sj = clamp_sp(species[jn], S.nsp);
  const double rcut = (S.radii[si] + S.radii[sj]) * S.rcutfac;
  PairGeomD PG;
  geom_hvp(S, rij[3 * p], rij[3 * p + 1], rij[3 * p + 2], v[3 * jn] - v[3 * i], v[3 * jn + 1] - v[3 * i + 1],
           v[3 * jn + 2] - v[3 * i + 2], rcut, S.weight[sj], PG);
  snapchain::Geom2 G;
  G.a = make_double2(PG.ar.v, PG.ai.v);
  G.at = make_double2(PG.ar.t, PG.ai.t);
  G.b = make_double2(PG.br.v, PG.bi.v);
  G.bt = make_double2(PG.br.t, PG.bi.t);
  Dual uk = PG.u[0];
  G.da = make_double2(PG.dar[0].v, PG.dai[0].v);
  G.dat = make_double2(PG.dar[0].t, PG.dai[0].t);
  G.db = make_double2(PG.dbr[0].v, PG.dbi[0].v);
  G.dbt = make_double2(PG.dbr[0].t, PG.dbi[0].t);
#pragma unroll
  for (int q = 1; q < 3; q++)  // direction k by selects (a runtime index would put PG in local memory)
    if (q == k) {
      uk = PG.u[q];
      G.da = make_double2(PG.dar[q].v, PG.dai[q].v);
      G.dat = make_double2(PG.dar[q].t, PG.dai[q].t);
      G.db = make_double2(PG.dbr[q].v, PG.dbi[q].v);
      G.dbt = make_double2(PG.dbr[q].t, PG.dbi[q].t);
    }
  double T[6];
  if (staged)
    snapchain::all_chains_hvp<J>(G, ysm + (i - first), ydm + (i - first), HVP_Y_ATOMS, T, save, HVP_T, threadIdx.x);
  else
    snapchain::all_chains_hvp<J>(G, Yw + i, Yd + i, natoms, T, save, HVP_T, threadIdx.x);
  const double cu = PG.dsfac.v * uk.v, cut = PG.dsfac.t * uk.v + PG.dsfac.v * uk.t;
  fdot[3 * p + k] = 2.0 * (cut * T[0] + cu * T[2] + PG.sfac.t * T[1] + PG.sfac.v * T[3] + cu * T[4] +
                           PG.sfac.v * T[5]);
}

// The Hessian-vector product of the pair forces from U and one tangent chain
// (snapchain::all_chains_hvp_lie), one thread per pair for all three directions: Yw and Ydot
// of up to HVP_LIE_ATOMS owners staged in shared memory (zero beyond each row's weighted
// entries), the start rows of U and its tangent saved per thread.  The pair geometry with its
// tangent is computed before the chains for (a, b) and again after them for the force
// coefficients, so that none of it is held in registers across the chains.
constexpr int HVP_LIE_T = 128;
constexpr int HVP_LIE_ATOMS = 8;
__host__ __device__ constexpr size_t hvp_lie_smem(int J, int uh) {
  return ((size_t)2 * (J + 1) * HVP_LIE_T + (size_t)2 * uh * HVP_LIE_ATOMS) * sizeof(double2);
}
__device__ __forceinline__ double opaque(double x) {  // the same value, not recognised as such
  double y;
  asm volatile("mov.b64 %0, %1;" : "=d"(y) : "d"(x));
  return y;
}
template <int J>
__global__ void __launch_bounds__(HVP_LIE_T) k_snap_pair_hvp_lie(const __grid_constant__ SnapDev S,
                                                                 const int64_t* __restrict__ d_np, int64_t natoms,
                                                                 const int32_t* __restrict__ owner,
                                                                 const int32_t* __restrict__ nbr,
                                                                 const double* __restrict__ rij,
                                                                 const int32_t* __restrict__ species,
                                                                 const double* __restrict__ v,
                                                                 const double2* __restrict__ Yw,
                                                                 const double2* __restrict__ Yd,
                                                                 double* __restrict__ fdot) {
  extern __shared__ double2 hsm[];  // save [2 (J+1)][HVP_LIE_T], then Yw, Yd [2][u_half][HVP_LIE_ATOMS]
  const int64_t np = *d_np;
  const int64_t p0 = (int64_t)blockIdx.x * blockDim.x, p = p0 + threadIdx.x;
  if (p0 >= np) return;  // block-uniform
  const int first = owner[p0];
  const int lastat = owner[(p0 + blockDim.x < np ? p0 + blockDim.x : np) - 1];
  const int UH = S.u_half;
  double2* ysm = hsm + 2 * (J + 1) * HVP_LIE_T;
  double2* ydm = ysm + UH * HVP_LIE_ATOMS;
  const int i = p < np ? owner[p] : -1;
  int32_t jn = 0;
  double rcut = 1.0, wj = 0.0, x = 1.0, y = 0.0, z = 0.0, tx = 0.0, ty = 0.0, tz = 0.0;
  double2 a = make_double2(1.0, 0.0), at = make_double2(0.0, 0.0), b = at, bt = at;
  if (p < np) {
    jn = nbr[p];
    const int si = clamp_sp(species[i], S.nsp), sj = clamp_sp(species[jn], S.nsp);
    rcut = (S.radii[si] + S.radii[sj]) * S.rcutfac;
    wj = S.weight[sj];
    x = rij[3 * p];
    y = rij[3 * p + 1];
    z = rij[3 * p + 2];
    tx = v[3 * jn] - v[3 * i];
    ty = v[3 * jn + 1] - v[3 * i + 1];
    tz = v[3 * jn + 2] - v[3 * i + 2];
    PairGeomD PG;
    geom_hvp(S, x, y, z, tx, ty, tz, rcut, wj, PG);
    a = make_double2(PG.ar.v, PG.ai.v);
    at = make_double2(PG.ar.t, PG.ai.t);
    b = make_double2(PG.br.v, PG.bi.v);
    bt = make_double2(PG.br.t, PG.bi.t);
  }
  double acc[12];
#pragma unroll
  for (int q = 0; q < 12; q++) acc[q] = 0.0;
  for (int g0 = first; g0 <= lastat; g0 += HVP_LIE_ATOMS) {  // block-uniform bounds
    const int nat = lastat - g0 + 1 < HVP_LIE_ATOMS ? lastat - g0 + 1 : HVP_LIE_ATOMS;
    if (g0 > first) __syncthreads();  // the previous group's readers are done
    for (int idx = threadIdx.x; idx < UH * nat; idx += blockDim.x) {
      const int h = idx / nat, at_ = idx - h * nat;
      const bool wt = (S.h_info[h] >> 16) != 0;  // the Y kernels leave the unweighted entries unset
      const size_t gi = (size_t)h * natoms + g0 + at_;
      ysm[h * HVP_LIE_ATOMS + at_] = wt ? Yw[gi] : make_double2(0.0, 0.0);
      ydm[h * HVP_LIE_ATOMS + at_] = wt ? Yd[gi] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    if (i >= g0 && i < g0 + nat)
      snapchain::all_chains_hvp_lie<J>(a, at, b, bt, ysm + (i - g0), ydm + (i - g0), HVP_LIE_ATOMS, acc, hsm,
                                       HVP_LIE_T, threadIdx.x);
  }
  if (p >= np) return;
  PairGeomD G;
  geom_hvp(S, opaque(x), opaque(y), opaque(z), opaque(tx), opaque(ty), opaque(tz), rcut, wj, G);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const Dual c0 = 2.0 * (G.dsfac * G.u[k]);
    const Dual f = 2.0 * G.sfac;
    const Dual c1 = f * (G.ai * G.dar[k] - G.ar * G.dai[k] + G.br * G.dbi[k] - G.bi * G.dbr[k]);
    const Dual c2 = f * (G.br * G.dar[k] + G.bi * G.dai[k] - G.ar * G.dbr[k] - G.ai * G.dbi[k]);
    const Dual c3 = f * (G.br * G.dai[k] - G.bi * G.dar[k] - G.ai * G.dbr[k] + G.ar * G.dbi[k]);
    fdot[3 * p + k] = c0.t * acc[0] + c0.v * (acc[1] + acc[2]) + (c1.t * acc[3] + c1.v * (acc[4] + acc[5])) +
                      (c2.t * acc[6] + c2.v * (acc[7] + acc[8])) + (c3.t * acc[9] + c3.v * (acc[10] + acc[11]));
  }
}

template <int J>
int launch_pair_hvp_lie_j(ipg_ctx* ctx, const SnapDev& S, int64_t np, const int64_t* d_np, int64_t natoms,
                          const int32_t* owner, const int32_t* nbr, const double* rij, const int32_t* species,
                          const double* v, const double2* Yw, const double2* Yd, double* fdot) {
  const size_t sm = hvp_lie_smem(J, S.u_half);
  if (sm > 48 * 1024)
    CUDA_RET(ctx, cudaFuncSetAttribute(k_snap_pair_hvp_lie<J>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  IPG_TIMED_LAUNCH(ctx, "snap_hvp", k_snap_pair_hvp_lie<J>, nblk(np, HVP_LIE_T), HVP_LIE_T, sm, S, d_np, natoms, owner,
                   nbr, rij, species, v, Yw, Yd, fdot);
  return IPG_OK;
}

template <int J>
int launch_pair_hvp_j(ipg_ctx* ctx, const SnapDev& S, int64_t np, const int64_t* d_np, int64_t natoms,
                      const int32_t* owner, const int32_t* nbr, const double* rij, const int32_t* species,
                      const double* v, const double2* Yw, const double2* Yd, double* fdot) {
  const size_t base = (size_t)4 * (J + 1) * HVP_T * sizeof(double2);
  const size_t with_y = base + (size_t)2 * S.u_half * HVP_Y_ATOMS * sizeof(double2);
  const int ystage = with_y <= 113 * 1024 ? HVP_Y_ATOMS : 0;  // two blocks per SM still fit
  const size_t sm = ystage ? with_y : base;
  if (sm > 48 * 1024)
    CUDA_RET(ctx, cudaFuncSetAttribute(k_snap_pair_hvp<J>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  const dim3 grid((unsigned)nblk(np, HVP_T), 3);
  IPG_TIMED_LAUNCH(ctx, "snap_hvp", k_snap_pair_hvp<J>, grid, HVP_T, sm, S, d_np, natoms, owner, nbr, rij, species,
                   v, Yw, Yd, fdot, ystage);
  return IPG_OK;
}

// tangent: the second-order tangent chains (k_snap_pair_hvp) instead of U and one tangent chain with
// the generator identity (k_snap_pair_hvp_lie)
int launch_pair_hvp(ipg_ctx* ctx, const SnapDev& S, int64_t np, const int64_t* d_np, int64_t natoms,
                    const int32_t* owner, const int32_t* nbr, const double* rij, const int32_t* species,
                    const double* v, const double2* Yw, const double2* Yd, double* fdot, bool tangent) {
  if (np == 0) return IPG_OK;
  switch (S.J) {
#define IPG_J(JJ) \
  case JJ:        \
    return tangent ? launch_pair_hvp_j<JJ>(ctx, S, np, d_np, natoms, owner, nbr, rij, species, v, Yw, Yd, fdot) \
                   : launch_pair_hvp_lie_j<JJ>(ctx, S, np, d_np, natoms, owner, nbr, rij, species, v, Yw, Yd, fdot);
    IPG_J(0) IPG_J(1) IPG_J(2) IPG_J(3) IPG_J(4) IPG_J(5) IPG_J(6) IPG_J(7) IPG_J(8)
#undef IPG_J
    default:
      return IPG_ERR_UNSUPPORTED;
  }
}

constexpr int PAIR_CHAIN_MAX_J = 10;  // twojmax handled by the register-chain kernel

template <int J, int MB>
int launch_chain(ipg_ctx* ctx, const SnapDev& S, int64_t np, const int64_t* d_np, int64_t natoms, const int32_t* owner,
                 const int32_t* nbr, const double* rij, const int32_t* species, const double2* Yw, double* part) {
  if constexpr (MB <= J / 2) {
    const int T = 128;
    IPG_TIMED_LAUNCH(ctx, "snap_pair", (k_snap_pair_adj<J, MB>), nblk(np, T), T, 0, S, d_np, natoms, owner, nbr, rij,
                     species, Yw, part);
    return launch_chain<J, MB + 1>(ctx, S, np, d_np, natoms, owner, nbr, rij, species, Yw, part);
  }
  return IPG_OK;
}

int launch_pair_adj(ipg_ctx* ctx, const SnapDev& S, int64_t np, const int64_t* d_np, int64_t natoms, const int32_t* owner,
                    const int32_t* nbr, const double* rij, const int32_t* species, const double2* Yw, double* part) {
  if (np == 0) return IPG_OK;
  switch (S.J) {
#define IPG_J(JJ) \
  case JJ:        \
    return launch_chain<JJ, 0>(ctx, S, np, d_np, natoms, owner, nbr, rij, species, Yw, part);
    IPG_J(0) IPG_J(1) IPG_J(2) IPG_J(3) IPG_J(4) IPG_J(5) IPG_J(6) IPG_J(7) IPG_J(8) IPG_J(9) IPG_J(10)
#undef IPG_J
    default:
      return IPG_ERR_UNSUPPORTED;
  }
}

// Plain path contraction: f_p = dB_i/dr_ij . beta[s_i] from the materialised dB/dr.
// fvec[p] = dbl[p] . beta of the pair's centre atom i: K components of dbl [np][K][3]; beta per
// atom (atom_stride > 0: beta + i*atom_stride) or per species (beta + s_i*sp_stride).
__global__ void k_snap_contract(int64_t n, const int64_t* __restrict__ off, const int32_t* __restrict__ species,
                                int nsp, const double* __restrict__ dbl, const double* __restrict__ beta, int K,
                                int64_t atom_stride, int64_t sp_stride, double* __restrict__ fvec) {
  // one warp per atom; lanes over (pair, component) rows
  int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (i >= n) return;
  const double* bt = atom_stride > 0 ? beta + (size_t)i * atom_stride : beta + (size_t)clamp_sp(species[i], nsp) * sp_stride;
  for (int64_t p = off[i]; p < off[i + 1]; p++) {
    const double* d = dbl + (size_t)p * K * 3;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int b = lane; b < K; b += 32) {
      double bb = bt[b];
      a0 += d[3 * b] * bb;
      a1 += d[3 * b + 1] * bb;
      a2 += d[3 * b + 2] * bb;
    }
    a0 = warp_sum(a0);
    a1 = warp_sum(a1);
    a2 = warp_sum(a2);
    if (lane == 0) {
      fvec[3 * p] = a0;
      fvec[3 * p + 1] = a1;
      fvec[3 * p + 2] = a2;
    }
  }
}

// F_k = sum_{p in out(k)} f_p - sum_{q in in(k)} f_q; per-atom virial contribution
// w6[k] = sum_{p in out(k)} f_p (x) (x_k - x_j(p)) with absolute positions
// (snap.jl:292-306 contracted with beta): [xx, yy, zz, yz, xz, xy] as in the reference.
__global__ void k_snap_gather(int64_t n, const int64_t* __restrict__ off, const int32_t* __restrict__ nbr,
                              const int64_t* __restrict__ in_off, const int64_t* __restrict__ in_pair,
                              const double* __restrict__ fvec, int nch, const double* __restrict__ pos,
                              double* __restrict__ F, double* __restrict__ w6) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double f0 = 0.0, f1 = 0.0, f2 = 0.0;
  double w[6] = {0, 0, 0, 0, 0, 0};
  const double xk = pos[3 * k], yk = pos[3 * k + 1], zk = pos[3 * k + 2];
  for (int64_t p = off[k]; p < off[k + 1]; p++) {
    double a = 0.0, b = 0.0, c = 0.0;
    for (int q = 0; q < nch; q++) {  // the chains' shares of this pair, in fixed order
      const double* fv = fvec + ((size_t)p * nch + q) * 3;
      a += fv[0];
      b += fv[1];
      c += fv[2];
    }
    f0 += a;
    f1 += b;
    f2 += c;
    int64_t jn = nbr[p];
    double dx = xk - pos[3 * jn], dy = yk - pos[3 * jn + 1], dz = zk - pos[3 * jn + 2];
    w[0] += a * dx;
    w[1] += b * dy;
    w[2] += c * dz;
    w[3] += b * dz;
    w[4] += a * dz;
    w[5] += a * dy;
  }
  for (int64_t q = in_off[k]; q < in_off[k + 1]; q++) {
    int64_t p = in_pair[q];
    double a = 0.0, b = 0.0, c = 0.0;
    for (int r = 0; r < nch; r++) {
      const double* fv = fvec + ((size_t)p * nch + r) * 3;
      a += fv[0];
      b += fv[1];
      c += fv[2];
    }
    f0 -= a;
    f1 -= b;
    f2 -= c;
  }
  if (F) {
    F[3 * k] = f0;
    F[3 * k + 1] = f1;
    F[3 * k + 2] = f2;
  }
  if (w6)
    for (int c = 0; c < 6; c++) w6[6 * k + c] = w[c];
}

// Per-configuration sums in fixed order: chunks of atoms (chunk table on the host:
// config, first atom, end) are reduced by one block each, then the chunks of each
// configuration are added in order: E[c] = beta0 + sum Ei, W6[c] = sum w6.
constexpr int RED_CHUNK = 1024;
__global__ void k_chunk_reduce(const int64_t* __restrict__ chunks, const double* __restrict__ Ei,
                               const double* __restrict__ w6, double* __restrict__ part) {
  __shared__ double sm[7][128];
  const int64_t a0 = chunks[3 * blockIdx.x + 1], a1 = chunks[3 * blockIdx.x + 2];
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int64_t i = a0 + threadIdx.x; i < a1; i += blockDim.x) {
    acc[0] += Ei ? Ei[i] : 0.0;
    if (w6)
      for (int q = 0; q < 6; q++) acc[1 + q] += w6[6 * i + q];
  }
  for (int q = 0; q < 7; q++) sm[q][threadIdx.x] = acc[q];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o)
      for (int q = 0; q < 7; q++) sm[q][threadIdx.x] += sm[q][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < 7) part[7 * blockIdx.x + threadIdx.x] = sm[threadIdx.x][0];
}

// One block of CONF_T threads per configuration: thread t sums chunks t, t + CONF_T, ... of
// its configuration, then a fixed-order tree over the threads.
constexpr int CONF_T = 64;
__global__ void __launch_bounds__(CONF_T) k_conf_reduce(int nconf, const int64_t* __restrict__ conf_chunk,
                                                        const double* __restrict__ part,
                                                        const double* __restrict__ beta0p, double* __restrict__ E,
                                                        double* __restrict__ W6) {
  __shared__ double sm[7][CONF_T];
  const int c = blockIdx.x;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int64_t k = conf_chunk[c] + threadIdx.x; k < conf_chunk[c + 1]; k += CONF_T)
    for (int q = 0; q < 7; q++) acc[q] += part[7 * k + q];
  for (int q = 0; q < 7; q++) sm[q][threadIdx.x] = acc[q];
  __syncthreads();
  for (int o = CONF_T / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o)
      for (int q = 0; q < 7; q++) sm[q][threadIdx.x] += sm[q][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0 && E) E[c] = *beta0p + sm[0][0];
  if (threadIdx.x < 6 && W6) W6[6 * c + threadIdx.x] = sm[1 + threadIdx.x][0];
}

// Per-atom force descriptors: dB_k[block s][b][c] = sum_{p in out(k), s_k = s} dbl_p -
// sum_{q in in(k), s_owner(q) = s} dbl_q   (snap.jl:289-290).  One thread per (atom, b*3+c).
__global__ void k_snap_dB_atoms(int64_t n, int K, int nsp, const int64_t* __restrict__ off,
                                const int64_t* __restrict__ in_off, const int64_t* __restrict__ in_pair,
                                const int32_t* __restrict__ owner, const int32_t* __restrict__ species,
                                const double* __restrict__ dbl, double* __restrict__ dB, int rows) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t k = t / (3 * K);
  int bc = (int)(t - k * 3 * K);
  if (k >= n) return;
  double acc[IPG_MAX_SNAP_SPECIES];
#pragma unroll
  for (int s = 0; s < IPG_MAX_SNAP_SPECIES; s++) acc[s] = 0.0;
  const int sk = species[k];
  double own = 0.0;
  for (int64_t p = off[k]; p < off[k + 1]; p++) own += dbl[(size_t)p * 3 * K + bc];
#pragma unroll
  for (int s = 0; s < IPG_MAX_SNAP_SPECIES; s++)
    if (s == sk) acc[s] += own;
  for (int64_t q = in_off[k]; q < in_off[k + 1]; q++) {
    int64_t p = in_pair[q];
    int so = species[owner[p]];
    double v = dbl[(size_t)p * 3 * K + bc];
#pragma unroll
    for (int s = 0; s < IPG_MAX_SNAP_SPECIES; s++)
      if (s == so) acc[s] -= v;
  }
  const int b = bc / 3, c = bc - 3 * b;
  if (rows)  // fitting layout: row 3k + c, column s*K + b
    for (int s = 0; s < nsp; s++) dB[((size_t)k * 3 + c) * K * nsp + (size_t)s * K + b] = acc[s];
  else
    for (int s = 0; s < nsp; s++) dB[((size_t)k * K * nsp + (size_t)s * K + b) * 3 + c] = acc[s];
}

// Fitting rows of each configuration (one block per configuration, threads over columns):
// Ae[c][s*K + k] = sum of B_i[k] over the atoms i of c with species s, and
// Aw[c][v][s*K + k] = W of the configuration's atoms (the k_snap_W_desc sum, snap.jl:267-281).
__global__ void k_snap_fit_rows(int nconf, const int64_t* __restrict__ conf_off, int K, int nsp,
                                const int32_t* __restrict__ species, const double* __restrict__ B,
                                const int64_t* __restrict__ off, const int32_t* __restrict__ nbr,
                                const double* __restrict__ pos, const double* __restrict__ dbl,
                                double* __restrict__ Ae, double* __restrict__ Aw) {
  const int c = blockIdx.x;
  if (c >= nconf) return;
  const int64_t a0 = conf_off[c], a1 = conf_off[c + 1];
  const int KN = K * nsp;
  for (int col = threadIdx.x; col < KN; col += blockDim.x) {
    const int sp = col / K, b = col - sp * K;
    if (Ae) {
      double e = 0.0;
      for (int64_t i = a0; i < a1; i++)
        if (clamp_sp(species[i], nsp) == sp) e += B[(size_t)i * K + b];
      Ae[(size_t)c * KN + col] = e;
    }
    if (Aw) {
      double w[6] = {0, 0, 0, 0, 0, 0};
      for (int64_t i = a0; i < a1; i++) {
        if (clamp_sp(species[i], nsp) != sp) continue;
        const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
        for (int64_t p = off[i]; p < off[i + 1]; p++) {
          const double* d = dbl + ((size_t)p * K + b) * 3;
          const int64_t jn = nbr[p];
          const double dx = xi - pos[3 * jn], dy = yi - pos[3 * jn + 1], dz = zi - pos[3 * jn + 2];
          w[0] += d[0] * dx;
          w[1] += d[1] * dy;
          w[2] += d[2] * dz;
          w[3] += d[1] * dz;
          w[4] += d[0] * dz;
          w[5] += d[0] * dy;
        }
      }
      for (int v = 0; v < 6; v++) Aw[((size_t)c * 6 + v) * KN + col] = w[v];
    }
  }
}

// owner[p] = the centre atom of pair p: one warp per atom, lanes over its pairs (coalesced).
__global__ void k_pair_owner(int64_t n, const int64_t* __restrict__ off, int32_t* __restrict__ owner) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= n) return;
  for (int64_t p = off[i] + (threadIdx.x & 31); p < off[i + 1]; p += 32) owner[p] = (int32_t)i;
}

// Virial descriptors W[block s][b][6] = sum over pairs of dB_i/dr_ij (x) (x_i - x_j)
// (snap.jl:292-306), per-block partials [grid][nsp*K*6].  Thread per component b,
// atoms strided over blocks.
__global__ void k_snap_W_desc(int64_t n, int K, int nsp, const int64_t* __restrict__ off,
                              const int32_t* __restrict__ nbr, const int32_t* __restrict__ species,
                              const double* __restrict__ pos, const double* __restrict__ dbl,
                              double* __restrict__ part) {
  extern __shared__ double wsm[];  // [nsp][K][6]
  for (int q = threadIdx.x; q < nsp * K * 6; q += blockDim.x) wsm[q] = 0.0;
  __syncthreads();
  for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
    const int s = clamp_sp(species[i], nsp);
    const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
    for (int b = threadIdx.x; b < K; b += blockDim.x) {
      double w[6] = {0, 0, 0, 0, 0, 0};
      for (int64_t p = off[i]; p < off[i + 1]; p++) {
        const double* d = dbl + ((size_t)p * K + b) * 3;
        int64_t jn = nbr[p];
        double dx = xi - pos[3 * jn], dy = yi - pos[3 * jn + 1], dz = zi - pos[3 * jn + 2];
        w[0] += d[0] * dx;
        w[1] += d[1] * dy;
        w[2] += d[2] * dz;
        w[3] += d[1] * dz;
        w[4] += d[0] * dz;
        w[5] += d[0] * dy;
      }
      for (int c = 0; c < 6; c++) wsm[((size_t)s * K + b) * 6 + c] += w[c];
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nsp * K * 6; q += blockDim.x) part[(size_t)blockIdx.x * nsp * K * 6 + q] = wsm[q];
}

// The W descriptors when their [nsp][K][6] sums do not fit shared memory (quadratic SNAP):
// one thread per component b sums every atom and pair in order, straight into W.
__global__ void k_snap_W_cols(int64_t n, int K, int nsp, const int64_t* __restrict__ off,
                              const int32_t* __restrict__ nbr, const int32_t* __restrict__ species,
                              const double* __restrict__ pos, const double* __restrict__ dbl, double* __restrict__ W) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= K) return;
  for (int s = 0; s < nsp; s++)
    for (int c = 0; c < 6; c++) W[((size_t)s * K + b) * 6 + c] = 0.0;
  for (int64_t i = 0; i < n; i++) {
    const int s = clamp_sp(species[i], nsp);
    const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
    double w[6] = {0, 0, 0, 0, 0, 0};
    for (int64_t p = off[i]; p < off[i + 1]; p++) {
      const double* d = dbl + ((size_t)p * K + b) * 3;
      const int64_t jn = nbr[p];
      const double dx = xi - pos[3 * jn], dy = yi - pos[3 * jn + 1], dz = zi - pos[3 * jn + 2];
      w[0] += d[0] * dx;
      w[1] += d[1] * dy;
      w[2] += d[2] * dz;
      w[3] += d[1] * dz;
      w[4] += d[0] * dz;
      w[5] += d[0] * dy;
    }
    for (int c = 0; c < 6; c++) W[((size_t)s * K + b) * 6 + c] += w[c];
  }
}

__global__ void k_sum_partials(int64_t nblocks, int width, const double* __restrict__ part, double* __restrict__ out,
                               double scale_add_base) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= width) return;
  double s = scale_add_base;
  for (int64_t b = 0; b < nblocks; b++) s += part[b * width + q];
  out[q] = s;
}

// Beta pullback from the descriptors (chem_flag / quadratic SNAP): block b sums the atoms of
// its contiguous range, threads over the (species block, component) columns:
// part[b][s][q] = sum_a [s_a = s] gE B_a[q] + g_a . dB_a[s K + q]  (dB_a [K*nsp][3]).
__global__ void k_gbeta_desc(int64_t n, int K, int nsp, const int32_t* __restrict__ species,
                             const double* __restrict__ B, const double* __restrict__ dB, const double* __restrict__ g,
                             double gE, double* __restrict__ part) {
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  const int64_t a0 = (int64_t)blockIdx.x * per, a1 = a0 + per < n ? a0 + per : n;
  const int KN = K * nsp;
  for (int col = threadIdx.x; col < KN; col += blockDim.x) {
    const int sp = col / K, q = col - sp * K;
    double acc = 0.0;
    for (int64_t a = a0; a < a1; a++) {
      if (species[a] == sp) acc += gE * B[(size_t)a * K + q];
      const double* d = dB + ((size_t)a * KN + col) * 3;
      acc += g[3 * a] * d[0] + g[3 * a + 1] * d[1] + g[3 * a + 2] * d[2];
    }
    part[(size_t)blockIdx.x * KN + col] = acc;
  }
}

// Per-block sums of x[0 .. n) over contiguous ranges of ceil(n / gridDim.x) items, each in a
// fixed order (blockDim.x = 256).
__global__ void k_sum_partials_strided(int64_t n, const double* __restrict__ x, double* __restrict__ out) {
  __shared__ double sm[256];
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  const int64_t b = (int64_t)blockIdx.x * per, e = b + per < n ? b + per : n;
  double v = 0.0;
  for (int64_t i = b + threadIdx.x; i < e; i += blockDim.x) v += x[i];
  sm[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = sm[0];
}

// ycoef[s][z] = y_mult[z] * beta[s][y_jjb[z]]
__global__ void k_ycoef(int nsp, int nz, int K, const double* __restrict__ ymult, const int32_t* __restrict__ yjjb,
                        const double* __restrict__ beta, double* __restrict__ ycoef) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nsp * nz) return;
  int s = t / nz, z = t - s * nz;
  ycoef[t] = ymult[z] * beta[(size_t)s * K + yjjb[z]];
}

// out = x + t u (3n coordinates).
// gpos = -gE F + Fdot: the position pullback d(gE E + gF . F)/dx = -gE F - H gF, with
// H gF = -Fdot the tangent of the forces along gF.
__global__ void k_vjp_pos(int64_t m, const double* __restrict__ F0, double gE, const double* __restrict__ Fdot,
                          double* __restrict__ gpos) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  double g = -gE * F0[k];
  if (Fdot) g += Fdot[k];
  gpos[k] = g;
}

// Elementwise loss pieces: g = 2 (F - F_ref), per-atom |F - F_ref|^2.
__global__ void k_loss_grad(int64_t n, const double* __restrict__ F, const double* __restrict__ Fref,
                            double* __restrict__ g, double* __restrict__ li) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int c = 0; c < 3; c++) {
    double d = F[3 * i + c] - Fref[3 * i + c];
    g[3 * i + c] = 2.0 * d;
    s += d * d;
  }
  li[i] = s;
}

}  // namespace

// ---------------------------------------------------------------------------------
struct ipg_snap {
  ipg_ctx* ctx = nullptr;
  ipg_snap_params p;
  SnapHost h;
  SnapDev dev;
  void* d_tables = nullptr;
  double* d_ymult = nullptr;
  int32_t* d_yjjb = nullptr;
  std::vector<double> cutsq;
  double radius = 0.0;
  int threads = 128;
  int blocks_per_sm = 0;  // 0 = occupancy-derived
  bool generic_adjoint = false;  // force the in-block per-neighbor adjoint (testing)
  std::vector<int64_t> chunk_tab;  // per-configuration reduction chunks (host staging)
  bool pair_split = false;  // adjoint pair kernel: one thread per (pair, chain) instead of per pair
  bool pair_tangent = false;  // adjoint pair kernel: forward tangent chains instead of the generator identity
  bool y_entries = false;   // Y kernel: one Z entry at a time (k_snap_yatoms) even where rows fit
  int utot_warps = 4;       // atoms (warps) per block of the per-chain Utot kernels
  bool utot_split = false;  // Utot: one launch per chain (k_snap_utot) instead of k_snap_utot_all
  int64_t vjp_chunk = 0;     // atoms per Z chunk (0: about 4 GiB of Z)
  bool generic_plain = false;  // plain path: the per-atom block kernel (IPG_GENERIC_PLAIN=1)
  bool generic_hvp = false;    // position pullback: the per-atom forward-mode kernel (IPG_GENERIC_HVP=1)
  int walk_warps = 4;       // atoms (warps) per block of the neighbor walk
  int yr_warps = 12;        // warps per block of the adjoint Y kernel (8, 10, 12 or 16)
  std::vector<double> beta_host;  // last uploaded beta
  // last evaluation's pair count, cell grids and chunk table (host), for graph capture
  int64_t last_np = 0;
  std::vector<ConfGrid> last_grid;
  std::vector<int64_t> last_chunks;
  // Captured batched evaluations (ipg_snap_batch_energy_forces_dev with graph != 0): the
  // key is everything the captured launches bake in (shape, boxes, mode, buffers).
  struct Graph {
    int32_t nconfig = 0;
    int mode = 0;
    std::vector<int64_t> off;
    std::vector<double> L;
    const void *pos = nullptr, *sp = nullptr;
    void *E = nullptr, *F = nullptr, *W6 = nullptr;
    const void* Fref = nullptr;  // training steps: F_ref, loss, dL/dbeta buffers
    void *loss = nullptr, *gbeta = nullptr;
    bool pair_split = false, y_entries = false;
    int utot_warps = 0, walk_warps = 0;
    cudaGraphExec_t exec = nullptr;
    uint64_t gen = 0;  // ctx->scratch_gen at capture
    int64_t cap = 0;   // pair capacity
    std::vector<ConfGrid> grid;
    std::vector<int64_t> chunks;
  };
  std::vector<Graph> graphs;
  int64_t graph_replays = 0;
  // Verlet-skin reuse of the neighbor list (ipg_snap_set_skin)
  double skin = 0.0;
  struct SkinCache {
    bool valid = false;
    int64_t n = 0;
    int nconf = 0;
    std::vector<int64_t> off;
    std::vector<double> L;
    CellList cl;      // buffers under the "skin_" prefix
    PairList pairs;   // the list with enlarged cutoffs
    double* ref = nullptr;     // positions at the build
    int32_t* ref_sp = nullptr;  // species at the build (a change rebuilds the list)
  } sk;
  int64_t skin_builds = 0, skin_reuses = 0;
};

namespace {

int upload_tables(ipg_snap* s) {
  ipg_ctx* ctx = s->ctx;
  SnapHost& h = s->h;
  // one allocation: rootpq | cglist | ymult (doubles), idxz | db (structs), y_off | y_jjz | yjjb (ints)
  auto pad = [](size_t b) { return (b + 255) & ~size_t(255); };
  size_t o_rpq = 0;
  size_t o_cg = o_rpq + pad(h.rootpq.size() * 8);
  size_t o_ym = o_cg + pad(h.cglist.size() * 8);
  size_t o_z = o_ym + pad(h.y_mult.size() * 8);
  size_t o_db = o_z + pad(h.idxz.size() * sizeof(ZDev));
  size_t o_yoff = o_db + pad(h.db.size() * sizeof(DBDev));
  size_t o_yjjz = o_yoff + pad(h.y_off.size() * 4);
  size_t o_yjjb = o_yjjz + pad(h.y_jjz.size() * 4);
  size_t o_zperm = o_yjjb + pad(h.y_jjb.size() * 4);
  size_t o_yso = o_zperm + pad(h.zperm.size() * 4);
  size_t o_ysh = o_yso + pad(h.ysched_off.size() * 4);
  size_t o_ysw = o_ysh + pad(h.ysched_h.size() * 4);
  size_t o_uoh = o_ysw + pad(h.ysched_w.size() * 8);
  size_t o_hinfo = o_uoh + pad(h.u_of_h.size() * 4);
  size_t o_hsgen = o_hinfo + pad(h.h_info.size() * 4);
  size_t o_yrows = o_hsgen + pad(h.h_sgen.size() * 8);
  size_t o_yit = o_yrows + pad(h.yrows.size() * sizeof(YRowDev));
  size_t o_yca = o_yit + pad(h.yitems.size() * sizeof(YItemDev));
  size_t o_ytj = o_yca + pad(h.yca.size() * 8);
  size_t total = o_ytj + pad(h.ytrip_jjz.size() * 4);
  CUDA_RET(ctx, cudaMalloc(&s->d_tables, total));
  char* b = static_cast<char*>(s->d_tables);
  std::vector<char> hostbuf(total, 0);
  memcpy(hostbuf.data() + o_rpq, h.rootpq.data(), h.rootpq.size() * 8);
  memcpy(hostbuf.data() + o_cg, h.cglist.data(), h.cglist.size() * 8);
  memcpy(hostbuf.data() + o_ym, h.y_mult.data(), h.y_mult.size() * 8);
  memcpy(hostbuf.data() + o_z, h.idxz.data(), h.idxz.size() * sizeof(ZDev));
  memcpy(hostbuf.data() + o_db, h.db.data(), h.db.size() * sizeof(DBDev));
  memcpy(hostbuf.data() + o_yoff, h.y_off.data(), h.y_off.size() * 4);
  memcpy(hostbuf.data() + o_yjjz, h.y_jjz.data(), h.y_jjz.size() * 4);
  memcpy(hostbuf.data() + o_yjjb, h.y_jjb.data(), h.y_jjb.size() * 4);
  memcpy(hostbuf.data() + o_zperm, h.zperm.data(), h.zperm.size() * 4);
  memcpy(hostbuf.data() + o_yso, h.ysched_off.data(), h.ysched_off.size() * 4);
  memcpy(hostbuf.data() + o_ysh, h.ysched_h.data(), h.ysched_h.size() * 4);
  memcpy(hostbuf.data() + o_ysw, h.ysched_w.data(), h.ysched_w.size() * 8);
  memcpy(hostbuf.data() + o_uoh, h.u_of_h.data(), h.u_of_h.size() * 4);
  memcpy(hostbuf.data() + o_hinfo, h.h_info.data(), h.h_info.size() * 4);
  memcpy(hostbuf.data() + o_hsgen, h.h_sgen.data(), h.h_sgen.size() * 8);
  memcpy(hostbuf.data() + o_yrows, h.yrows.data(), h.yrows.size() * sizeof(YRowDev));
  memcpy(hostbuf.data() + o_yit, h.yitems.data(), h.yitems.size() * sizeof(YItemDev));
  memcpy(hostbuf.data() + o_yca, h.yca.data(), h.yca.size() * 8);
  memcpy(hostbuf.data() + o_ytj, h.ytrip_jjz.data(), h.ytrip_jjz.size() * 4);
  CUDA_RET(ctx, cudaMemcpy(b, hostbuf.data(), total, cudaMemcpyHostToDevice));
  SnapDev& d = s->dev;
  memset(&d, 0, sizeof(d));
  d.J = h.J;
  d.nsp = s->p.nspecies;
  d.chem = s->p.chem_flag ? 1 : 0;
  d.nelem = d.chem ? s->p.nspecies : 1;
  d.wselfall = s->p.wselfall_flag ? 1 : 0;
  d.literal_chem_z = s->p.literal_chem_z ? 1 : 0;
  d.quadratic = s->p.quadratic_flag ? 1 : 0;
  d.klin = h.idxb_max * d.nelem * d.nelem * d.nelem;
  d.K = d.quadratic ? d.klin + d.klin * (d.klin + 1) / 2 : d.klin;
  d.idxu_max = h.idxu_max;
  d.idxz_max = h.idxz_max;
  d.u_half = h.u_half;
  d.ext_max = h.ext_max;
  d.idxcg_max = h.idxcg_max;
  d.switch_flag = s->p.switch_flag;
  d.bzero_flag = s->p.bzero_flag;
  d.bnorm_flag = s->p.bnorm_flag;
  d.rcutfac = s->p.rcutfac;
  d.rmin0 = s->p.rmin0;
  d.rfac0 = s->p.rfac0;
  d.wself = 1.0;
  for (int q = 0; q < s->p.nspecies; q++) {
    d.radii[q] = s->p.radii[q];
    d.weight[q] = s->p.weight[q];
  }
  for (int j = 0; j <= h.J; j++) {
    d.idxu_block[j] = h.idxu_block[j];
    d.bzero[j] = h.bzero[j];
  }
  for (int j = 0; j <= h.J + 1; j++) d.half_block[j] = h.half_block[j];
  d.rootpq = reinterpret_cast<const double*>(b + o_rpq);
  d.cglist = reinterpret_cast<const double*>(b + o_cg);
  d.idxz = reinterpret_cast<const ZDev*>(b + o_z);
  d.db = reinterpret_cast<const DBDev*>(b + o_db);
  d.y_off = reinterpret_cast<const int32_t*>(b + o_yoff);
  d.y_jjz = reinterpret_cast<const int32_t*>(b + o_yjjz);
  d.zperm = reinterpret_cast<const int32_t*>(b + o_zperm);
  d.ysched_off = reinterpret_cast<const int32_t*>(b + o_yso);
  d.ysched_h = reinterpret_cast<const int32_t*>(b + o_ysh);
  d.ysched_w = reinterpret_cast<const double*>(b + o_ysw);
  d.u_of_h = reinterpret_cast<const int32_t*>(b + o_uoh);
  d.h_info = reinterpret_cast<const int32_t*>(b + o_hinfo);
  d.h_sgen = reinterpret_cast<const double2*>(b + o_hsgen);
  d.n_yrows = (int)h.yrows.size();
  d.yrows = reinterpret_cast<const YRowDev*>(b + o_yrows);
  d.yitems = reinterpret_cast<const YItemDev*>(b + o_yit);
  d.yca = reinterpret_cast<const double*>(b + o_yca);
  d.ytrip_jjz = reinterpret_cast<const int32_t*>(b + o_ytj);
  d.n_ytrip = (int)h.ytrip_jjz.size();
  d.n_yca = (int)h.yca.size();
  s->d_ymult = reinterpret_cast<double*>(b + o_ym);
  s->d_yjjb = reinterpret_cast<int32_t*>(b + o_yjjb);
  return IPG_OK;
}

template <int MODE>
int launch_atoms(ipg_snap* s, const SnapDev& dev, const SnapIO& io, int64_t natoms, int64_t* grid_used) {
  ipg_ctx* ctx = s->ctx;
  const bool levels = needs_levels(MODE, io.utot_in != nullptr, io.yout != nullptr);
  const int threads = levels ? s->threads : 256;
  SmemLayout L = smem_layout(dev, threads / 32, MODE, levels);
  size_t smem = L.total;
  if (smem > 227 * 1024)
    return ipg_fail(ctx, IPG_ERR_UNSUPPORTED, "twojmax %d needs %zu bytes of shared memory per block", dev.J, smem);
  CUDA_RET(ctx, cudaFuncSetAttribute(k_snap_atom<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = s->blocks_per_sm;
  if (per_sm <= 0) {
    CUDA_RET(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_snap_atom<MODE>, threads, smem));
    per_sm = std::max(1, per_sm);
  }
  int64_t grid = std::min<int64_t>(std::max<int64_t>(natoms, 1), (int64_t)ctx->num_sms * per_sm);
  if (grid_used) *grid_used = grid;
  IPG_TIMED_LAUNCH(ctx, "snap_atom", k_snap_atom<MODE>, (unsigned)grid, threads, smem, dev, io);
  return IPG_OK;
}

// Uploads beta [nsp][K], the energy shifts and beta0 (device: beta | ebias[8] | beta0) and
// the per-Z-entry Y coefficients; while a graph is being captured only the pointers are
// set (the replay path uploads before each launch).
int set_beta(ipg_snap* s, const double* beta, double beta0, SnapDev& dev) {
  ipg_ctx* ctx = s->ctx;
  const int K = dev.K, nsp = s->p.nspecies;
  const bool chemq = dev.chem || dev.quadratic;  // bzero is inside B there: no energy shift
  double *d_beta, *d_ycoef;
  const size_t nb = (size_t)nsp * K;
  IPG_RET(scratch(ctx, "snap_beta", nb + IPG_MAX_SNAP_SPECIES + 1, &d_beta));
  IPG_RET(scratch(ctx, "snap_ycoef", (size_t)nsp * s->h.idxz_max, &d_ycoef));
  dev.beta = d_beta;
  dev.ycoef = d_ycoef;
  dev.ebias = d_beta + nb;
  dev.beta0 = d_beta + nb + IPG_MAX_SNAP_SPECIES;
  if (ctx->capturing) return IPG_OK;
  double* hb = host_scratch<double>(ctx, "snap_beta_h", nb + IPG_MAX_SNAP_SPECIES + 1);
  for (size_t k = 0; k < nb; k++) hb[k] = beta ? beta[k] : 0.0;
  for (int q = 0; q < IPG_MAX_SNAP_SPECIES; q++) {  // -beta[s] . bzero[j(k)] (compute_b.jl:134-155)
    double t = 0.0;
    if (q < nsp && !chemq)
      for (int k = 0; k < K; k++) t += hb[(size_t)q * K + k] * s->h.bzero[s->h.idxb[3 * k + 2]];
    hb[nb + q] = -t;
  }
  hb[nb + IPG_MAX_SNAP_SPECIES] = beta0;
  CUDA_RET(ctx, cudaMemcpyAsync(d_beta, hb, (nb + IPG_MAX_SNAP_SPECIES + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
  IPG_LAUNCH(ctx, k_ycoef, nblk((int64_t)nsp * s->h.idxz_max, 256), 256, 0, nsp, s->h.idxz_max, K, s->d_ymult,
             s->d_yjjb, d_beta, d_ycoef);
  return IPG_OK;
}

int snap_neighbors_inner(ipg_snap* s, int64_t n, const double* d_pos, const int32_t* d_species, int nconf,
                         const int64_t* h_atom_off, const double* h_L, PairList& pl, int64_t cap);

// Neighbor build for a set of configurations (device positions); cap > 0: capacity mode.
int snap_neighbors(ipg_snap* s, int64_t n, const double* d_pos, const int32_t* d_species, int nconf,
                   const int64_t* h_atom_off, const double* h_L, PairList& pl, int64_t cap = 0) {
  IPG_RET(ipg_timing_mark(s->ctx, "neighbor", true));
  int st = snap_neighbors_inner(s, n, d_pos, d_species, nconf, h_atom_off, h_L, pl, cap);
  if (st) return st;
  return ipg_timing_mark(s->ctx, "neighbor", false);
}

int snap_neighbors_inner(ipg_snap* s, int64_t n, const double* d_pos, const int32_t* d_species, int nconf,
                         const int64_t* h_atom_off, const double* h_L, PairList& pl, int64_t cap) {
  const int mode_sk = IPG_NLIST_FULL | (s->p.literal_sqrt_radius ? IPG_NLIST_LITERAL_SQRT : 0);
  if (s->skin > 0.0 && cap == 0 && !s->ctx->capturing && n > 0 && !s->p.literal_sqrt_radius) {
    // Verlet skin: reuse the list built with cutoffs + skin while no atom has moved more
    // than skin/2 since that build (then every pair now within a cutoff is in it)
    ipg_snap::SkinCache& C = s->sk;
    bool valid = C.valid && C.n == n && C.nconf == nconf &&
                 memcmp(C.off.data(), h_atom_off, sizeof(int64_t) * (nconf + 1)) == 0 &&
                 memcmp(C.L.data(), h_L, sizeof(double) * 3 * nconf) == 0;
    if (valid) {
      double d2;
      IPG_RET(ipg_max_disp2(s->ctx, C.cl, d_pos, C.ref, d_species, C.ref_sp, &d2));
      valid = d2 <= 0.25 * s->skin * s->skin;
    }
    if (!valid) {
      const int nsp = s->p.nspecies;
      std::vector<double> cut2(nsp * nsp);
      for (int q = 0; q < nsp * nsp; q++) {
        const double r = std::sqrt(s->cutsq[q]) + s->skin;
        cut2[q] = r * r;
      }
      IPG_RET(ipg_build_cells(s->ctx, "skin_", n, d_pos, d_species, nsp, nconf, h_atom_off, h_L,
                              s->radius + s->skin, C.cl));
      IPG_RET(ipg_build_pairs(s->ctx, "skin_", C.cl, d_species, nsp, cut2.data(), IPG_NLIST_FULL, false, C.pairs,
                              false, 0, s->walk_warps));
      IPG_RET(scratch(s->ctx, "skin_ref", 3 * (size_t)n, &C.ref));
      IPG_RET(scratch(s->ctx, "skin_ref_sp", (size_t)n, &C.ref_sp));
      CUDA_RET(s->ctx, cudaMemcpyAsync(C.ref, d_pos, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice,
                                       s->ctx->stream));
      CUDA_RET(s->ctx, cudaMemcpyAsync(C.ref_sp, d_species, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice,
                                       s->ctx->stream));
      C.valid = true;
      C.n = n;
      C.nconf = nconf;
      C.off.assign(h_atom_off, h_atom_off + nconf + 1);
      C.L.assign(h_L, h_L + 3 * nconf);
      s->skin_builds++;
    } else {
      s->skin_reuses++;
    }
    s->last_grid = C.cl.h_grid;
    return ipg_filter_pairs(s->ctx, "snap_", C.cl, C.pairs, d_pos, d_species, s->p.nspecies, s->cutsq.data(),
                            mode_sk, pl);
  }
  CellList cl;
  IPG_RET(ipg_build_cells(s->ctx, "snap_", n, d_pos, d_species, s->p.nspecies, nconf, h_atom_off, h_L, s->radius,
                          cl));
  s->last_grid = cl.h_grid;
  int mode = IPG_NLIST_FULL | (s->p.literal_sqrt_radius ? IPG_NLIST_LITERAL_SQRT : 0);
  IPG_RET(ipg_build_pairs(s->ctx, "snap_", cl, d_species, s->p.nspecies, s->cutsq.data(), mode, true, pl, false,
                          cap, s->walk_warps));
  return IPG_OK;
}

struct EvalOut {
  double* E = nullptr;   // [nconf] device
  double* F = nullptr;   // [3n] device
  double* W6 = nullptr;  // [nconf][6] device
  double* B = nullptr;   // [n][K] device
  double* dB = nullptr;  // [n][K*nsp][3] device ([3n][K*nsp] with dB_rows)
  double* Wd = nullptr;  // [K*nsp][6] device
  bool dB_rows = false;
  double* Ae = nullptr;  // [nconf][K*nsp] fitting energy rows (device)
  double* Aw = nullptr;  // [nconf][6][K*nsp] fitting virial rows (device)
  PairList* pl_out = nullptr;          // receives the pair list (stays valid until the next build)
  const double2** utot_out = nullptr;  // receives Utot [n][idxu_max] when the chain kernel made it
  const double2** yw_out = nullptr;    // adjoint mode: receives the weighted Y [u_half][n] of the chain path
  double2* zall = nullptr;  // adjoint mode: also write Z [idxz_max][n] here (row-blocked Y kernel only)
  bool* zall_done = nullptr;  // set when zall was written
};

// Atoms per chunk of the Z buffer (idxz_max entries per atom): about 4 GiB, or IPG_VJP_CHUNK.
int64_t zrows_chunk(const ipg_snap* s, const SnapDev& dev, int64_t n) {
  const int64_t zbytes = (int64_t)dev.idxz_max * (int64_t)sizeof(double2);
  int64_t C = std::max<int64_t>(YS_ATOMS, (((int64_t)4 << 30) / zbytes) / YS_ATOMS * YS_ATOMS);
  if (s->vjp_chunk > 0) C = std::max<int64_t>(YS_ATOMS, s->vjp_chunk / YS_ATOMS * YS_ATOMS);
  return std::max<int64_t>(1, std::min(C, n));
}

// Shared memory and blocks per SM of k_snap_yrows<YM_Z>.
int zrows_config(ipg_ctx* ctx, const SnapDev& dev, int* ysm, int* per_sm) {
  *ysm = yr_smem(dev.J, dev.nsp, dev.n_ytrip, dev.n_yca, dev.u_half, dev.n_yrows).total();
  CUDA_RET(ctx, cudaFuncSetAttribute(k_snap_yrows<YM_Z>, cudaFuncAttributeMaxDynamicSharedMemorySize, *ysm));
  *per_sm = 1;
  CUDA_RET(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_snap_yrows<YM_Z>, YS_WARPS * 32, *ysm));
  return IPG_OK;
}

// Plain dB/dr path on the register chains: per chunk of atoms, Z (row-blocked kernel), B and
// E_i (k_snap_bdesc), then dbl of the pairs those atoms own (k_snap_dbfused).
int plain_chains(ipg_snap* s, const SnapDev& dev, int64_t n, const PairList& pl, const int32_t* d_species,
                 const double2* utot, double* B, double* Ei, double* dbl) {
  ipg_ctx* ctx = s->ctx;
  const int64_t C = zrows_chunk(s, dev, n);
  double2* Z;
  IPG_RET(scratch(ctx, "snap_Z", (size_t)C * dev.idxz_max + 1, &Z));
  int ysm, yper;
  IPG_RET(zrows_config(ctx, dev, &ysm, &yper));
  const int bsm = (int)((size_t)dev.u_half * YS_ATOMS * sizeof(double2) + (size_t)dev.K * YS_ATOMS * 8);
  CUDA_RET(ctx, cudaFuncSetAttribute(k_snap_bdesc, cudaFuncAttributeMaxDynamicSharedMemorySize, bsm));
  int bper = 1;
  CUDA_RET(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bper, k_snap_bdesc, GB_WARPS * 32, bsm));
  for (int64_t a0 = 0; a0 < n; a0 += C) {
    const int64_t nc = std::min(C, n - a0);
    const int64_t tiles = (nc + YS_ATOMS - 1) / YS_ATOMS;
    const int64_t yg = std::min<int64_t>(tiles, (int64_t)ctx->num_sms * std::max(1, yper));
    IPG_TIMED_LAUNCH(ctx, "snap_zrows", k_snap_yrows<YM_Z>, (unsigned)yg, YS_WARPS * 32, ysm, dev, s->h.yconst, nc,
                     d_species + a0, utot + (size_t)a0 * dev.idxu_max, Z, (double*)nullptr, (double2*)nullptr);
    const int64_t bg = std::min<int64_t>(tiles, (int64_t)ctx->num_sms * std::max(1, bper));
    IPG_TIMED_LAUNCH(ctx, "snap_bdesc", k_snap_bdesc, (unsigned)bg, GB_WARPS * 32, bsm, dev, a0, nc, d_species, Z,
                     utot, B, Ei);
    IPG_RET(plain_fused(ctx, dev, a0, a0 + nc, pl.d_off, pl.d_j, pl.d_r, d_species, a0, nc, Z, dbl));
  }
  return IPG_OK;
}

// The Y kernel on the Utot of n atoms (full layout [n][idxu_max]): yout = weighted Y
// [u_half][n] and Ei = the energy of each atom; zall (optional) also receives Z (and
// *zall_done is set).  *done stays false when neither atoms-in-lanes kernel fits (the caller
// runs the generic per-atom kernel).  tname: the timing name of the launch.
int launch_y(ipg_snap* s, const SnapDev& dev, const char* tname, int64_t n, const int32_t* d_species,
             const double2* utot, double2* yout, double* Ei, double2* zall, bool* zall_done, bool* done) {
  ipg_ctx* ctx = s->ctx;
  *done = false;
  size_t ysm = (size_t)dev.u_half * YS_ATOMS * sizeof(double2);
  if (n == 0 || ysm > 200 * 1024) return IPG_OK;  // atoms-in-lanes: the Utot of 32 atoms in shared memory
  const bool rows = dev.J <= YR_MAX_J && !s->y_entries && s->h.yconst_ok;
  const bool withz = rows && zall;
  // warps per block of the Y-only kernel (IPG_YR_WARPS: 8, 10, 12 or 16)
  const int yw = rows && !withz ? s->yr_warps : YS_WARPS;
  const int ythreads = yw * 32;
  const void* kfn = !rows       ? (const void*)k_snap_yatoms
                    : withz     ? (const void*)k_snap_yrows<YM_YZ>
                    : yw == 10  ? (const void*)k_snap_yrows<YM_Y, 10>
                    : yw == 12  ? (const void*)k_snap_yrows<YM_Y, 12>
                    : yw == 16  ? (const void*)k_snap_yrows<YM_Y, 16>
                                : (const void*)k_snap_yrows<YM_Y>;
  if (rows) ysm = yr_smem(dev.J, dev.nsp, dev.n_ytrip, dev.n_yca, dev.u_half, dev.n_yrows).total();
  CUDA_RET(ctx, cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ysm));
  int per_sm = 1;
  CUDA_RET(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, ythreads, ysm));
  const int64_t groups = (n + YS_ATOMS - 1) / YS_ATOMS;
  const int64_t grid = std::min<int64_t>(groups, (int64_t)ctx->num_sms * std::max(1, per_sm));
  if (withz) {
    IPG_TIMED_LAUNCH(ctx, tname, k_snap_yrows<YM_YZ>, (unsigned)grid, ythreads, ysm, dev, s->h.yconst, n, d_species,
                     utot, yout, Ei, zall);
    if (zall_done) *zall_done = true;
  } else if (rows && yw == 10) {
    IPG_TIMED_LAUNCH(ctx, tname, (k_snap_yrows<YM_Y, 10>), (unsigned)grid, ythreads, ysm, dev, s->h.yconst, n,
                     d_species, utot, yout, Ei, (double2*)nullptr);
  } else if (rows && yw == 12) {
    IPG_TIMED_LAUNCH(ctx, tname, (k_snap_yrows<YM_Y, 12>), (unsigned)grid, ythreads, ysm, dev, s->h.yconst, n,
                     d_species, utot, yout, Ei, (double2*)nullptr);
  } else if (rows && yw == 16) {
    IPG_TIMED_LAUNCH(ctx, tname, (k_snap_yrows<YM_Y, 16>), (unsigned)grid, ythreads, ysm, dev, s->h.yconst, n,
                     d_species, utot, yout, Ei, (double2*)nullptr);
  } else if (rows) {
    IPG_TIMED_LAUNCH(ctx, tname, k_snap_yrows<YM_Y>, (unsigned)grid, ythreads, ysm, dev, s->h.yconst, n, d_species,
                     utot, yout, Ei, (double2*)nullptr);
  } else {
    IPG_TIMED_LAUNCH(ctx, tname, k_snap_yatoms, (unsigned)grid, ythreads, ysm, dev, n, d_species, utot, yout, Ei);
  }
  *done = true;
  return IPG_OK;
}

// Energy / forces / descriptors for device inputs.  mode: MODE_DESC (B/E only), MODE_ADJ,
// MODE_PLAIN.  Writes device outputs; does not synchronise.
int snap_eval(ipg_snap* s, int64_t n, const double* d_pos, const int32_t* d_species, int nconf,
              const int64_t* h_atom_off, const double* h_L, const double* beta, double beta0, int mode,
              const EvalOut& out, int64_t cap = 0) {
  ipg_ctx* ctx = s->ctx;
  SnapDev dev = s->dev;
  IPG_RET(set_beta(s, beta, beta0, dev));
  PairList pl;
  IPG_RET(snap_neighbors(s, n, d_pos, d_species, nconf, h_atom_off, h_L, pl, cap));
  const int K = dev.K, nsp = dev.nsp;
  const int64_t np = pl.npairs;
  if (cap == 0) s->last_np = np;
  double *Ei, *fvec = nullptr, *dbl = nullptr, *w6 = nullptr;
  IPG_RET(scratch(ctx, "snap_Ei", (size_t)n + 1, &Ei));
  SnapIO io;
  memset(&io, 0, sizeof(io));
  io.n = n;
  io.off = pl.d_off;
  io.nbr = pl.d_j;
  io.rij = pl.d_r;
  io.species = d_species;
  io.Ei = Ei;
  io.B = out.B;
  io.status = ctx->d_status;
  const bool need_plain = (mode == MODE_PLAIN) || out.dB || out.Wd || out.Aw;
  const bool chemq = dev.chem || dev.quadratic;  // element-resolved / quadratic SNAP kernel
  const bool chains = dev.J <= PAIR_CHAIN_MAX_J && !s->generic_adjoint && !chemq;
  if (chains && n) {  // Utot from the register-chain kernel
    double2* utot;
    IPG_RET(scratch(ctx, "snap_utot", (size_t)n * dev.idxu_max + 1, &utot));
    IPG_RET(launch_utot(ctx, dev, n, pl.d_off, pl.d_j, pl.d_r, d_species, utot, s->utot_warps, !s->utot_split));
    io.utot_in = utot;
  }
  int nch = 1;
  if (chemq) {
    // chem_flag / quadratic_flag: B (and E_i), and dB_lin/dr of every pair when forces or
    // force descriptors are wanted; the forces contract dB/dr with beta (quadratic: with each
    // atom's effective linear coefficients), the descriptors read the extended dB/dr.
    const int KL = dev.klin;
    const bool forces = mode != MODE_DESC && (out.F || out.W6);
    const bool want_db = out.dB || out.Wd || out.Aw;
    const bool plain = forces || want_db;
    double* Bx = out.B;
    if (dev.quadratic && want_db && !Bx) IPG_RET(scratch(ctx, "snap_Bx", (size_t)n * K + 1, &Bx));
    io.B = Bx;
    double *dlin = nullptr, *beff = nullptr;
    if (plain) IPG_RET(scratch(ctx, "snap_dbl", (size_t)np * KL * 3 + 3, &dlin));
    if (dev.quadratic && forces) IPG_RET(scratch(ctx, "snap_beff", (size_t)n * KL + 1, &beff));
    io.dbl = dlin;
    const ChemSmem CL = chem_smem(dev, 4, plain);
    if (CL.total > 227 * 1024)
      return ipg_fail(ctx, IPG_ERR_UNSUPPORTED, "chem/quadratic SNAP needs %zu bytes of shared memory", CL.total);
    const void* kfn = plain ? (const void*)k_snap_chem<true> : (const void*)k_snap_chem<false>;
    CUDA_RET(ctx, cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CL.total));
    int per_sm = 1;
    CUDA_RET(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, 128, CL.total));
    const int64_t grid = std::min<int64_t>(std::max<int64_t>(n, 1), (int64_t)ctx->num_sms * std::max(1, per_sm));
    double2* zbuf;
    IPG_RET(scratch(ctx, "snap_chem_z", (size_t)grid * dev.nelem * dev.nelem * dev.idxz_max + 1, &zbuf));
    if (n) {
      if (plain)
        IPG_TIMED_LAUNCH(ctx, "snap_atom", k_snap_chem<true>, (unsigned)grid, 128, CL.total, dev, io, zbuf, beff);
      else
        IPG_TIMED_LAUNCH(ctx, "snap_atom", k_snap_chem<false>, (unsigned)grid, 128, CL.total, dev, io, zbuf, beff);
    }
    if (forces) {
      IPG_RET(scratch(ctx, "snap_fvec", 3 * (size_t)np + 3, &fvec));
      if (n)
        IPG_TIMED_LAUNCH(ctx, "snap_contract", k_snap_contract, nblk(32 * n, 256), 256, 0, n, pl.d_off, d_species, nsp,
                         dlin, beff ? beff : dev.beta, KL, beff ? (int64_t)KL : (int64_t)0, (int64_t)K, fvec);
    }
    if (want_db) {
      dbl = dlin;
      if (dev.quadratic) {  // the extended dB/dr of every pair
        int32_t* owner;
        IPG_RET(scratch(ctx, "snap_owner", (size_t)np + 1, &owner));
        IPG_RET(scratch(ctx, "snap_dbx", (size_t)np * K * 3 + 3, &dbl));
        if (n) {
          IPG_LAUNCH(ctx, k_pair_owner, nblk(32 * n, 256), 256, 0, n, pl.d_off, owner);
          IPG_LAUNCH(ctx, k_quad_pairs, nblk(np * KL, 256), 256, 0, np, pl.d_np, KL, K, owner, Bx, dlin, dbl);
        }
      }
    }
  } else if (mode == MODE_ADJ && chains) {
    // per-atom kernel writes the weighted Y; the register-chain kernel does the neighbors
    nch = s->pair_split ? dev.J / 2 + 1 : 1;
    double2* yout;
    int32_t* owner;
    IPG_RET(scratch(ctx, "snap_yout", (size_t)n * dev.u_half + 1, &yout));
    IPG_RET(scratch(ctx, "snap_owner", (size_t)np + 1, &owner));
    IPG_RET(scratch(ctx, "snap_fvec", 3 * (size_t)np * nch + 3, &fvec));
    io.yout = yout;
    if (n) {
      IPG_LAUNCH(ctx, k_pair_owner, nblk(32 * n, 256), 256, 0, n, pl.d_off, owner);
      bool ydone = false;
      IPG_RET(launch_y(s, dev, "snap_atom", n, d_species, io.utot_in, yout, Ei, out.zall, out.zall_done, &ydone));
      if (!ydone) IPG_RET(launch_atoms<MODE_ADJY>(s, dev, io, n, nullptr));
      if (out.yw_out) *out.yw_out = yout;
      if (s->pair_split)
        IPG_RET(launch_pair_adj(ctx, dev, np, pl.d_np, n, owner, pl.d_j, pl.d_r, d_species, yout, fvec));
      else if (s->pair_tangent)
        IPG_RET(launch_pair_adj_all(ctx, dev, np, pl.d_np, n, owner, pl.d_j, pl.d_r, d_species, yout, fvec));
      else
        IPG_RET(launch_pair_lie(ctx, dev, np, pl.d_np, n, owner, pl.d_j, pl.d_r, d_species, yout, fvec));
    }
  } else if (mode == MODE_ADJ) {
    IPG_RET(scratch(ctx, "snap_fvec", 3 * (size_t)np + 3, &fvec));
    io.fvec = fvec;
    if (n) IPG_RET(launch_atoms<MODE_ADJ>(s, dev, io, n, nullptr));
  } else if (need_plain) {
    IPG_RET(scratch(ctx, "snap_dbl", (size_t)np * K * 3 + 3, &dbl));
    io.dbl = dbl;
    if (n && chains && dev.J <= YR_MAX_J && s->h.yconst_ok && cap == 0 && !s->generic_plain)
      IPG_RET(plain_chains(s, dev, n, pl, d_species, io.utot_in, out.B, Ei, dbl));
    else if (n)
      IPG_RET(launch_atoms<MODE_PLAIN>(s, dev, io, n, nullptr));
    if (out.F || out.W6) {
      IPG_RET(scratch(ctx, "snap_fvec", 3 * (size_t)np + 3, &fvec));
      if (n) IPG_TIMED_LAUNCH(ctx, "snap_contract", k_snap_contract, nblk(32 * n, 256), 256, 0, n, pl.d_off, d_species, nsp, dbl, dev.beta, K,
                               (int64_t)0, (int64_t)K, fvec);
    }
  } else if (chains && n && dev.J <= YR_MAX_J && s->h.yconst_ok && cap == 0) {
    // Z from the row-blocked kernel per chunk of atoms, then B (and E_i) per atom tile
    const int64_t C = zrows_chunk(s, dev, n);
    double2* Z;
    IPG_RET(scratch(ctx, "snap_Z", (size_t)C * dev.idxz_max + 1, &Z));
    int ysm, yper;
    IPG_RET(zrows_config(ctx, dev, &ysm, &yper));
    const int bsm = (int)((size_t)dev.u_half * YS_ATOMS * sizeof(double2) + (size_t)K * YS_ATOMS * 8);
    CUDA_RET(ctx, cudaFuncSetAttribute(k_snap_bdesc, cudaFuncAttributeMaxDynamicSharedMemorySize, bsm));
    int bper = 1;
    CUDA_RET(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bper, k_snap_bdesc, GB_WARPS * 32, bsm));
    for (int64_t a0 = 0; a0 < n; a0 += C) {
      const int64_t nc = std::min(C, n - a0);
      const int64_t tiles = (nc + YS_ATOMS - 1) / YS_ATOMS;
      const int64_t yg = std::min<int64_t>(tiles, (int64_t)ctx->num_sms * std::max(1, yper));
      IPG_TIMED_LAUNCH(ctx, "snap_zrows", k_snap_yrows<YM_Z>, (unsigned)yg, YS_WARPS * 32, ysm, dev, s->h.yconst, nc,
                       d_species + a0, io.utot_in + (size_t)a0 * dev.idxu_max, Z, (double*)nullptr, (double2*)nullptr);
      const int64_t bg = std::min<int64_t>(tiles, (int64_t)ctx->num_sms * std::max(1, bper));
      IPG_TIMED_LAUNCH(ctx, "snap_bdesc", k_snap_bdesc, (unsigned)bg, GB_WARPS * 32, bsm, dev, a0, nc, d_species, Z,
                       io.utot_in, out.B, Ei);
    }
  } else {
    if (n) IPG_RET(launch_atoms<MODE_DESC>(s, dev, io, n, nullptr));
  }
  if (out.W6) IPG_RET(scratch(ctx, "snap_w6", 6 * (size_t)n + 6, &w6));
  IPG_RET(ipg_side_join(ctx));  // the list transpose (side stream) is read from here on
  if ((out.F || out.W6) && fvec && n)
    IPG_TIMED_LAUNCH(ctx, "snap_gather", k_snap_gather, nblk(n, 128), 128, 0, n, pl.d_off, pl.d_j, pl.d_in_off,
                     pl.d_in_pair, fvec, nch, d_pos, out.F, w6);
  if (out.E || out.W6) {
    // chunk table: [config, first atom, end] per chunk, then each config's chunk range
    std::vector<int64_t>& ch = s->chunk_tab;
    ch.clear();
    std::vector<int64_t> cc(nconf + 1, 0);
    for (int c = 0; c < nconf; c++) {
      int64_t a = h_atom_off[c], b = h_atom_off[c + 1];
      if (a == b) {
        ch.insert(ch.end(), {c, a, a});
      }
      for (int64_t x = a; x < b; x += RED_CHUNK) ch.insert(ch.end(), {c, x, std::min(b, x + RED_CHUNK)});
      cc[c + 1] = (int64_t)ch.size() / 3;
    }
    const int64_t nchunk = (int64_t)ch.size() / 3;
    int64_t *d_ch, *d_cc;
    double* part;
    IPG_RET(scratch(ctx, "snap_chunks", ch.size() + cc.size(), &d_ch));
    IPG_RET(scratch(ctx, "snap_chunk_part", 7 * (size_t)nchunk, &part));
    int64_t* hb = host_scratch<int64_t>(ctx, "snap_chunks_h", ch.size() + cc.size());
    memcpy(hb, ch.data(), sizeof(int64_t) * ch.size());
    memcpy(hb + ch.size(), cc.data(), sizeof(int64_t) * cc.size());
    s->last_chunks.assign(hb, hb + ch.size() + cc.size());
    if (!ctx->capturing)  // a captured graph's chunk table is uploaded before each replay
      CUDA_RET(ctx, cudaMemcpyAsync(d_ch, hb, sizeof(int64_t) * (ch.size() + cc.size()), cudaMemcpyHostToDevice,
                                    ctx->stream));
    d_cc = d_ch + ch.size();
    IPG_LAUNCH(ctx, k_chunk_reduce, (unsigned)nchunk, 128, 0, d_ch, Ei, w6, part);
    if (nconf > 0)
      IPG_LAUNCH(ctx, k_conf_reduce, (unsigned)nconf, CONF_T, 0, nconf, d_cc, part, dev.beta0, out.E, out.W6);
  }
  if (out.dB && n) {
    int32_t* owner;
    IPG_RET(scratch(ctx, "snap_owner", (size_t)np + 1, &owner));
    IPG_LAUNCH(ctx, k_pair_owner, nblk(32 * n, 256), 256, 0, n, pl.d_off, owner);
    IPG_LAUNCH(ctx, k_snap_dB_atoms, nblk(n * 3 * K, 128), 128, 0, n, K, nsp, pl.d_off, pl.d_in_off, pl.d_in_pair,
               owner, d_species, dbl, out.dB, out.dB_rows ? 1 : 0);
  }
  if ((out.Ae || out.Aw) && n) {
    int64_t* d_coff;
    IPG_RET(scratch(ctx, "snap_fit_off", (size_t)nconf + 1, &d_coff));
    CUDA_RET(ctx, cudaMemcpyAsync(d_coff, h_atom_off, sizeof(int64_t) * (nconf + 1), cudaMemcpyHostToDevice,
                                  ctx->stream));
    IPG_LAUNCH(ctx, k_snap_fit_rows, (unsigned)nconf, 128, 0, nconf, d_coff, K, nsp, d_species, out.B, pl.d_off,
               pl.d_j, d_pos, dbl, out.Ae, out.Aw);
  }
  if (out.Wd && (size_t)nsp * K * 6 * 8 > 200 * 1024) {
    IPG_LAUNCH(ctx, k_snap_W_cols, nblk(K, 128), 128, 0, n, K, nsp, pl.d_off, pl.d_j, d_species, d_pos, dbl, out.Wd);
  } else if (out.Wd) {
    const int width = nsp * K * 6;
    int64_t grid = std::min<int64_t>(std::max<int64_t>(n, 1), 2 * ctx->num_sms);
    double* part;
    IPG_RET(scratch(ctx, "snap_wpart", (size_t)grid * width, &part));
    size_t sm = (size_t)width * 8;
    if (sm > 48 * 1024)
      CUDA_RET(ctx, cudaFuncSetAttribute(k_snap_W_desc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    IPG_LAUNCH(ctx, k_snap_W_desc, (unsigned)grid, 64, sm, n, K, nsp, pl.d_off, pl.d_j, d_species, d_pos, dbl, part);
    IPG_LAUNCH(ctx, k_sum_partials, nblk(width, 128), 128, 0, grid, width, part, out.Wd, 0.0);
  }
  if (out.pl_out) *out.pl_out = pl;
  if (out.utot_out) *out.utot_out = io.utot_in;
  return ipg_side_join(ctx);
}

int snap_vjp_device(ipg_snap* s, int64_t n, const double* d_pos, const int32_t* d_species, int nconf,
                    const int64_t* h_atom_off, const double* h_L, const double* beta, double gE, const double* d_g,
                    double* d_gbeta, const PairList* reuse_pl, const double2* reuse_utot, const double2* reuse_Z,
                    const double2** v_out = nullptr);

// Graph mode of a whole force-matching training step (snap_train_step).
constexpr int MODE_TRAIN = 100;
// Z of a training step is kept for the pullback when it takes at most this many bytes.
constexpr size_t TRAIN_Z_MAX = size_t(48) << 30;

// One force-matching training step over a batch (the fitting loop of PotentialLearning over
// the descriptors of src/BasisSystems/LAMMPS_SNAP/bispectrum.jl:279-387):
//   E, F, W6 of the adjoint path (o; F is required), L = sum_atoms |F - F_ref|^2 (d_loss) and
//   dL/dbeta = the beta pullback with cotangent 2 (F - F_ref) (d_gbeta [nspecies][K]).
// The pullback reuses the evaluation's pair list and Utot, and the Z the Y kernel wrote beside
// Y (when it fits TRAIN_Z_MAX).  Device buffers only, no synchronisation, so the whole step can
// be captured as one CUDA graph (cap > 0: capacity mode, as snap_eval).
int snap_train_step(ipg_snap* s, int64_t n, const double* d_pos, const int32_t* d_sp, int nconf, const int64_t* off,
                    const double* L, const double* beta, double beta0, const double* d_Fref, const EvalOut& o,
                    double* d_loss, double* d_gbeta, int64_t cap) {
  ipg_ctx* ctx = s->ctx;
  const SnapDev& dev = s->dev;
  double *d_g, *d_li, *d_lpart;
  IPG_RET(scratch(ctx, "loss_g", 3 * (size_t)n + 3, &d_g));
  IPG_RET(scratch(ctx, "loss_li", (size_t)n + 1, &d_li));
  const int64_t lblk = std::max<int64_t>(1, std::min<int64_t>((n + 1023) / 1024, 4096));
  IPG_RET(scratch(ctx, "loss_part", (size_t)lblk, &d_lpart));
  EvalOut oo = o;
  PairList pl;
  const double2* utot = nullptr;
  oo.pl_out = &pl;
  oo.utot_out = &utot;
  double2* Z = nullptr;
  bool zdone = false;
  const bool chains = dev.J <= PAIR_CHAIN_MAX_J && !s->generic_adjoint && !dev.chem && !dev.quadratic;
  if (chains && dev.J <= YR_MAX_J && s->h.yconst_ok && !s->y_entries && n &&
      (size_t)n * dev.idxz_max * sizeof(double2) <= TRAIN_Z_MAX) {
    IPG_RET(scratch(ctx, "train_Z", (size_t)n * dev.idxz_max + 1, &Z));
    oo.zall = Z;
    oo.zall_done = &zdone;
  }
  IPG_RET(snap_eval(s, n, d_pos, d_sp, nconf, off, L, beta, beta0, MODE_ADJ, oo, cap));
  if (n) {
    IPG_LAUNCH(ctx, k_loss_grad, nblk(n, 256), 256, 0, n, o.F, d_Fref, d_g, d_li);
    IPG_LAUNCH(ctx, k_sum_partials_strided, (unsigned)lblk, 256, 0, n, d_li, d_lpart);
    IPG_LAUNCH(ctx, k_sum_partials, 1, 32, 0, lblk, 1, d_lpart, d_loss, 0.0);
  } else {
    CUDA_RET(ctx, cudaMemsetAsync(d_loss, 0, sizeof(double), ctx->stream));
  }
  return snap_vjp_device(s, n, d_pos, d_sp, nconf, off, L, beta, 0.0, d_g, d_gbeta, &pl, utot, zdone ? Z : nullptr);
}

// ---- CUDA-graph replay of batched evaluations -------------------------------------------

// The device buffers of a force-matching training step (MODE_TRAIN graphs).
struct TrainBufs {
  const double* Fref = nullptr;
  double* loss = nullptr;
  double* gbeta = nullptr;
};

ipg_snap::Graph* find_graph(ipg_snap* s, int32_t nconfig, const int64_t* off, const double* L, int mode,
                            const void* pos, const void* sp, const EvalOut& o, const TrainBufs& tb) {
  for (auto& g : s->graphs) {
    if (g.nconfig != nconfig || g.mode != mode || g.pos != pos || g.sp != sp || g.E != o.E || g.F != o.F ||
        g.W6 != o.W6 || g.Fref != tb.Fref || g.loss != tb.loss || g.gbeta != tb.gbeta ||
        g.pair_split != s->pair_split || g.y_entries != s->y_entries ||
        g.utot_warps != s->utot_warps || g.walk_warps != s->walk_warps)
      continue;
    if (memcmp(g.off.data(), off, sizeof(int64_t) * (nconfig + 1)) != 0) continue;
    if (memcmp(g.L.data(), L, sizeof(double) * 3 * nconfig) != 0) continue;
    return &g;
  }
  return nullptr;
}

void drop_graph(ipg_snap* s, ipg_snap::Graph* g) {
  if (g->exec) cudaGraphExecDestroy(g->exec);
  s->graphs.erase(s->graphs.begin() + (g - s->graphs.data()));
}

// Replays the graph captured for this key: beta, the cell grids and the chunk table are
// uploaded first (the graph reads them from the same buffers), then one graph launch.
// Returns IPG_ERR_NOT_CAPTURED when there is no usable graph, IPG_ERR_CAPACITY when the
// pair count outgrew the captured capacity (the graph is dropped; the caller re-runs).
int batch_graph_replay(ipg_snap* s, int32_t nconfig, const int64_t* off, const double* d_pos, const int32_t* d_sp,
                       const double* L, const double* beta, double beta0, int mode, const EvalOut& o,
                       const TrainBufs& tb = TrainBufs()) {
  ipg_ctx* ctx = s->ctx;
  ipg_snap::Graph* g = find_graph(s, nconfig, off, L, mode, d_pos, d_sp, o, tb);
  if (!g) return IPG_ERR_NOT_CAPTURED;
  if (g->gen != ctx->scratch_gen) {  // a scratch buffer moved since the capture
    drop_graph(s, g);
    return IPG_ERR_NOT_CAPTURED;
  }
  SnapDev dev = s->dev;
  IPG_RET(set_beta(s, beta, beta0, dev));
  ConfGrid* d_grid;
  int64_t* d_ch;
  IPG_RET(scratch(ctx, "snap_grid", g->grid.size(), &d_grid));
  IPG_RET(scratch(ctx, "snap_chunks", g->chunks.size(), &d_ch));
  if (g->gen != ctx->scratch_gen) {  // set_beta or the lookups above had to allocate
    drop_graph(s, g);
    return IPG_ERR_NOT_CAPTURED;
  }
  CUDA_RET(ctx, cudaMemcpyAsync(d_grid, g->grid.data(), sizeof(ConfGrid) * g->grid.size(), cudaMemcpyHostToDevice,
                                ctx->stream));
  CUDA_RET(ctx, cudaMemcpyAsync(d_ch, g->chunks.data(), sizeof(int64_t) * g->chunks.size(), cudaMemcpyHostToDevice,
                                ctx->stream));
  IPG_RET(ipg_status_reset(ctx));
  CUDA_RET(ctx, cudaGraphLaunch(g->exec, ctx->stream));
  s->graph_replays++;
  int st = ipg_status_check(ctx, "ipg_snap_batch_energy_forces_dev (graph)");
  if (st == IPG_ERR_CAPACITY) drop_graph(s, g);
  return st;
}

// Captures the evaluation just run eagerly (same inputs) for later replays.  The pair
// buffers get 25% headroom over the count just seen; a warm run in capacity mode sizes
// every scratch buffer first, so nothing allocates while capturing.  Failures only mean
// that later calls run eagerly.
void batch_graph_capture(ipg_snap* s, int32_t nconfig, const int64_t* off, const double* d_pos, const int32_t* d_sp,
                         const double* L, const double* beta, double beta0, int mode, const EvalOut& o,
                         const TrainBufs& tb = TrainBufs()) {
  ipg_ctx* ctx = s->ctx;
  const int64_t n = off[nconfig];
  const int64_t cap = s->last_np + s->last_np / 4 + 1024;
  auto body = [&]() {
    return mode == MODE_TRAIN ? snap_train_step(s, n, d_pos, d_sp, nconfig, off, L, beta, beta0, tb.Fref, o, tb.loss,
                                                tb.gbeta, cap)
                              : snap_eval(s, n, d_pos, d_sp, nconfig, off, L, beta, beta0, mode, o, cap);
  };
  if (ipg_status_reset(ctx) || body() || ipg_status_check(ctx, "graph warm-up")) return;
  if (s->graphs.size() >= 8) drop_graph(s, &s->graphs.front());
  ipg_snap::Graph g;
  g.nconfig = nconfig;
  g.mode = mode;
  g.off.assign(off, off + nconfig + 1);
  g.L.assign(L, L + 3 * nconfig);
  g.pos = d_pos;
  g.sp = d_sp;
  g.E = o.E;
  g.F = o.F;
  g.W6 = o.W6;
  g.Fref = tb.Fref;
  g.loss = tb.loss;
  g.gbeta = tb.gbeta;
  g.pair_split = s->pair_split;
  g.y_entries = s->y_entries;
  g.utot_warps = s->utot_warps;
  g.walk_warps = s->walk_warps;
  g.cap = cap;
  g.grid = s->last_grid;
  g.chunks = s->last_chunks;
  const bool timing = ctx->timing;
  ctx->timing = false;
  ctx->capturing = true;
  cudaGraph_t graph = nullptr;
  int st = IPG_OK;
  if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
    st = IPG_ERR_CUDA;
  } else {
    st = body();
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    if (st == IPG_OK && e != cudaSuccess) st = IPG_ERR_CUDA;
  }
  ctx->capturing = false;
  ctx->timing = timing;
  if (st == IPG_OK && graph && cudaGraphInstantiate(&g.exec, graph, 0) == cudaSuccess) {
    g.gen = ctx->scratch_gen;
    s->graphs.push_back(std::move(g));
  }
  if (graph) cudaGraphDestroy(graph);
  cudaGetLastError();  // a failed capture leaves no sticky error behind
}

// ---- autotuner ------------------------------------------------------------------------
struct TuneChoice {
  int y_entries = 0, pair_split = 0, utot_split = 0, utot_warps = 4, walk_warps = 4;
  double ms = 0.0;
};

void tune_apply(ipg_snap* s, const TuneChoice& c) {
  s->y_entries = c.y_entries != 0;
  s->pair_split = c.pair_split != 0;
  s->utot_split = c.utot_split != 0;
  s->utot_warps = c.utot_warps;
  s->walk_warps = c.walk_warps;
}

int json_int(const std::string& line, const char* field, int dflt) {
  const std::string f = std::string("\"") + field + "\":";
  const size_t k = line.find(f);
  if (k == std::string::npos) return dflt;
  return atoi(line.c_str() + k + f.size());
}

// Cache: one JSON object per line; the last line with the key wins.
bool tune_cache_lookup(const char* path, const std::string& key, TuneChoice& c) {
  FILE* f = fopen(path, "r");
  if (!f) return false;
  bool hit = false;
  char buf[1024];
  const std::string want = "\"key\": \"" + key + "\"";
  while (fgets(buf, sizeof(buf), f)) {
    const std::string line(buf);
    if (line.find(want) == std::string::npos) continue;
    c.y_entries = json_int(line, "y_entries", 0);
    c.pair_split = json_int(line, "pair_split", 0);
    c.utot_split = json_int(line, "utot_split", 0);
    c.utot_warps = std::max(1, std::min(4, json_int(line, "utot_warps", 4)));
    c.walk_warps = std::max(1, std::min(4, json_int(line, "walk_warps", 4)));
    hit = true;
  }
  fclose(f);
  return hit;
}

std::string tune_json(const std::string& key, const TuneChoice& c, bool cached, int tried) {
  char buf[768];
  snprintf(buf, sizeof(buf),
           "{\"key\": \"%s\", \"y_entries\": %d, \"pair_split\": %d, \"utot_split\": %d, \"utot_warps\": %d, "
           "\"walk_warps\": %d, \"ms\": %.4f, \"cached\": %d, \"tried\": %d}",
           key.c_str(), c.y_entries, c.pair_split, c.utot_split, c.utot_warps, c.walk_warps, c.ms, cached ? 1 : 0,
           tried);
  return buf;
}

int check_common(ipg_snap* s, int64_t n, const void* pos, const void* species, const double* L) {
  if (!s) return IPG_ERR_ARG;
  if (n < 0 || n >= INT32_MAX) return ipg_fail(s->ctx, IPG_ERR_ARG, "n out of range");
  if (n > 0 && (!pos || !species)) return ipg_fail(s->ctx, IPG_ERR_ARG, "null positions or species");
  if (!L) return ipg_fail(s->ctx, IPG_ERR_ARG, "null box");
  return IPG_OK;
}

int check_offsets(ipg_ctx* ctx, int32_t nconfig, const int64_t* atom_offsets) {
  if (atom_offsets[0] != 0) return ipg_fail(ctx, IPG_ERR_ARG, "atom_offsets[0] must be 0");
  for (int c = 0; c < nconfig; c++)
    if (atom_offsets[c + 1] < atom_offsets[c]) return ipg_fail(ctx, IPG_ERR_ARG, "atom_offsets must be non-decreasing");
  return IPG_OK;
}

int check_host_inputs(ipg_snap* s, int64_t n, const double* pos, const int32_t* species) {
  if (!host_all_finite(pos, 3 * n)) return ipg_fail(s->ctx, IPG_ERR_NONFINITE, "non-finite position");
  if (!host_species_ok(species, n, s->p.nspecies))
    return ipg_fail(s->ctx, IPG_ERR_SPECIES, "species id out of range");
  return IPG_OK;
}

int upload_inputs(ipg_snap* s, int64_t n, const double* pos, const int32_t* species, double** d_pos,
                  int32_t** d_sp) {
  ipg_ctx* ctx = s->ctx;
  IPG_RET(scratch(ctx, "snap_in_pos", 3 * (size_t)n + 3, d_pos));
  IPG_RET(scratch(ctx, "snap_in_sp", (size_t)n + 1, d_sp));
  if (n) {
    IPG_RET(ipg_copy_h2d(ctx, *d_pos, pos, sizeof(double) * 3 * n));
    IPG_RET(ipg_copy_h2d(ctx, *d_sp, species, sizeof(int32_t) * n));
  }
  return IPG_OK;
}

}  // namespace

// ---------------------------------------------------------------------------------
extern "C" {

int ipg_snap_create(ipg_ctx* ctx, const ipg_snap_params* params, ipg_snap** out) {
  if (!ctx || !params || !out) return IPG_ERR_ARG;
  *out = nullptr;
  const ipg_snap_params& p = *params;
  if (p.twojmax < 0 || p.twojmax > SNAP_MAX_J)
    return ipg_fail(ctx, IPG_ERR_UNSUPPORTED, "twojmax must be in 0..%d", SNAP_MAX_J);
  if (p.nspecies < 1 || p.nspecies > IPG_MAX_SNAP_SPECIES)
    return ipg_fail(ctx, IPG_ERR_ARG, "nspecies must be in 1..%d", IPG_MAX_SNAP_SPECIES);
  if (p.chem_flag != p.bnorm_flag)  // snap.jl:10-13
    return ipg_fail(ctx, IPG_ERR_ARG, "chem_flag and bnorm_flag should be the same");
  if (!(p.rcutfac > 0.0)) return ipg_fail(ctx, IPG_ERR_ARG, "rcutfac must be > 0");
  for (int q = 0; q < p.nspecies; q++)
    if (!(p.radii[q] > 0.0)) return ipg_fail(ctx, IPG_ERR_ARG, "radii must be > 0");
  CUDA_RET(ctx, cudaSetDevice(ctx->device));
  ipg_snap* s = new ipg_snap();
  s->ctx = ctx;
  s->p = p;
  if (snap_build_tables(p, s->h) != IPG_OK) {
    delete s;
    return ipg_fail(ctx, IPG_ERR_ARG, "bad SNAP parameters");
  }
  int st = upload_tables(s);
  if (st) {
    delete s;
    return st;
  }
  {  // rootpq table of the register-chain kernel (independent of twojmax)
    constexpr int R = snapchain::RPQ_STRIDE;
    double t[R * R] = {};
    for (int a = 1; a < R; a++)
      for (int b = 1; b < R; b++) t[a * R + b] = std::sqrt((double)a / (double)b);
    cudaError_t e = cudaMemcpyToSymbol(snapchain::c_rpq, t, sizeof(t));
    // generator factors sqrt((m + 1)(j - m)) of the derivative identity
    constexpr int NR = snapchain::SGEN_ROWS;
    double t2[R * NR * R] = {};
    for (int j = 1; j < R; j++)
      for (int mb = 0; mb < NR; mb++)
        for (int m = 0; m < j; m++) t2[(j * NR + mb) * R + m] = std::sqrt((double)((m + 1) * (j - m)));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(snapchain::c_sgen, t2, sizeof(t2));
    if (e != cudaSuccess) {
      cudaFree(s->d_tables);
      delete s;
      return ipg_cuda_check(ctx, e, "rootpq upload");
    }
  }
  if (const char* g = getenv("IPG_GENERIC_ADJOINT")) s->generic_adjoint = g[0] == '1';
  if (const char* g = getenv("IPG_PAIR_SPLIT")) s->pair_split = g[0] == '1';
  if (const char* g = getenv("IPG_PAIR_TANGENT")) s->pair_tangent = g[0] == '1';
  if (const char* g = getenv("IPG_Y_ENTRIES")) s->y_entries = g[0] == '1';
  if (const char* g = getenv("IPG_UTOT_SPLIT")) s->utot_split = g[0] == '1';
  if (const char* g = getenv("IPG_VJP_CHUNK")) s->vjp_chunk = std::max<int64_t>(0, atoll(g));
  if (const char* g = getenv("IPG_GENERIC_PLAIN")) s->generic_plain = g[0] == '1';
  if (const char* g = getenv("IPG_GENERIC_HVP")) s->generic_hvp = g[0] == '1';
  if (const char* g = getenv("IPG_YR_WARPS")) {
    const int w = atoi(g);
    s->yr_warps = (w == 8 || w == 10 || w == 16) ? w : 12;
  }
  // cutoffs, utl.jl:41-56
  const int ns = p.nspecies;
  s->cutsq.assign(ns * ns, 0.0);
  double cutmax = 0.0;
  for (int a = 0; a < ns; a++) {
    double cut = 2.0 * p.radii[a] * p.rcutfac;
    cutmax = std::max(cutmax, cut);
    s->cutsq[a * ns + a] = cut * cut;
    for (int b = a + 1; b < ns; b++) {
      double c = (p.radii[a] + p.radii[b]) * p.rcutfac;
      s->cutsq[a * ns + b] = c * c;
      s->cutsq[b * ns + a] = c * c;
    }
  }
  s->radius = p.literal_sqrt_radius ? std::sqrt(cutmax) : cutmax;
  *out = s;
  return IPG_OK;
}

int ipg_snap_destroy(ipg_snap* s) {
  if (!s) return IPG_ERR_ARG;
  cudaSetDevice(s->ctx->device);
  cudaStreamSynchronize(s->ctx->stream);
  for (auto& g : s->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  if (s->d_tables) cudaFree(s->d_tables);
  delete s;
  return IPG_OK;
}

int ipg_snap_ncoeff(const ipg_snap* s, int32_t* K) {
  if (!s || !K) return IPG_ERR_ARG;
  *K = s->dev.K;
  return IPG_OK;
}

int ipg_snap_descriptors(ipg_snap* s, int64_t n, const double* pos, const int32_t* species, const double L[3],
                         double* B, double* dB, double* W, uint32_t what) {
  IPG_RET(check_common(s, n, pos, species, L));
  ipg_ctx* ctx = s->ctx;
  if (((what & IPG_DESC_B) && !B) || ((what & IPG_DESC_DB) && !dB && n) || ((what & IPG_DESC_W) && !W))
    return ipg_fail(ctx, IPG_ERR_ARG, "requested descriptor output is NULL");
  CUDA_RET(ctx, cudaSetDevice(ctx->device));
  IPG_RET(check_host_inputs(s, n, pos, species));
  double* d_pos;
  int32_t* d_sp;
  IPG_RET(upload_inputs(s, n, pos, species, &d_pos, &d_sp));
  IPG_RET(ipg_status_reset(ctx));
  const int K = s->dev.K, nsp = s->p.nspecies;
  EvalOut o;
  double *dB_d = nullptr, *B_d = nullptr, *W_d = nullptr;
  if (what & IPG_DESC_B) IPG_RET(scratch(ctx, "snap_out_B", (size_t)n * K + 1, &B_d));
  if (what & IPG_DESC_DB) IPG_RET(scratch(ctx, "snap_out_dB", (size_t)n * K * nsp * 3 + 1, &dB_d));
  if (what & IPG_DESC_W) IPG_RET(scratch(ctx, "snap_out_W", (size_t)K * nsp * 6 + 1, &W_d));
  o.B = B_d;
  o.dB = dB_d;
  o.Wd = W_d;
  int64_t aoff[2] = {0, n};
  IPG_RET(snap_eval(s, n, d_pos, d_sp, 1, aoff, L, nullptr, 0.0, MODE_DESC, o));
  if (B_d && n) IPG_RET(ipg_copy_d2h(ctx, B, B_d, sizeof(double) * n * K));
  if (dB_d && n) IPG_RET(ipg_copy_d2h(ctx, dB, dB_d, sizeof(double) * n * K * nsp * 3));
  if (W_d) {
    if (n) CUDA_RET(ctx, cudaMemcpyAsync(W, W_d, sizeof(double) * K * nsp * 6, cudaMemcpyDeviceToHost, ctx->stream));
    else memset(W, 0, sizeof(double) * K * nsp * 6);
  }
  return ipg_status_check(ctx, "ipg_snap_descriptors");
}

int ipg_snap_set_skin(ipg_snap* s, double skin) {
  if (!s) return IPG_ERR_ARG;
  if (!(skin >= 0.0) || !std::isfinite(skin)) return ipg_fail(s->ctx, IPG_ERR_ARG, "skin must be finite and >= 0");
  s->skin = skin;
  s->sk.valid = false;
  return IPG_OK;
}

int ipg_snap_skin_stats(const ipg_snap* s, int64_t* builds, int64_t* reuses) {
  if (!s) return IPG_ERR_ARG;
  if (builds) *builds = s->skin_builds;
  if (reuses) *reuses = s->skin_reuses;
  return IPG_OK;
}

int ipg_snap_batch_descriptors(ipg_snap* s, int32_t nconfig, const int64_t* atom_offsets, const double* pos,
                               const int32_t* species, const double* L, double* Ae, double* Af, double* Aw) {
  if (!s || nconfig < 1 || !atom_offsets || !L) return s ? ipg_fail(s->ctx, IPG_ERR_ARG, "bad batch args") : IPG_ERR_ARG;
  ipg_ctx* ctx = s->ctx;
  if (atom_offsets[0] != 0) return ipg_fail(ctx, IPG_ERR_ARG, "atom_offsets[0] must be 0");
  for (int c = 0; c < nconfig; c++)
    if (atom_offsets[c + 1] < atom_offsets[c]) return ipg_fail(ctx, IPG_ERR_ARG, "atom_offsets must be non-decreasing");
  const int64_t n = atom_offsets[nconfig];
  IPG_RET(check_common(s, n, pos, species, L));
  CUDA_RET(ctx, cudaSetDevice(ctx->device));
  IPG_RET(check_host_inputs(s, n, pos, species));
  double* d_pos;
  int32_t* d_sp;
  IPG_RET(upload_inputs(s, n, pos, species, &d_pos, &d_sp));
  const int K = s->dev.K, nsp = s->p.nspecies;
  const size_t KN = (size_t)K * nsp;
  double *B_d, *Ae_d = nullptr, *Af_d = nullptr, *Aw_d = nullptr;
  IPG_RET(scratch(ctx, "fit_B", (size_t)n * K + 1, &B_d));
  if (Ae) IPG_RET(scratch(ctx, "fit_Ae", (size_t)nconfig * KN, &Ae_d));
  if (Af) IPG_RET(scratch(ctx, "fit_Af", 3 * (size_t)n * KN + 1, &Af_d));
  if (Aw) IPG_RET(scratch(ctx, "fit_Aw", 6 * (size_t)nconfig * KN, &Aw_d));
  IPG_RET(ipg_status_reset(ctx));
  EvalOut o;
  o.B = B_d;
  o.dB = Af_d;
  o.dB_rows = true;
  o.Ae = Ae_d;
  o.Aw = Aw_d;
  IPG_RET(snap_eval(s, n, d_pos, d_sp, nconfig, atom_offsets, L, nullptr, 0.0, MODE_DESC, o));
  if (Ae) {
    if (n) CUDA_RET(ctx, cudaMemcpyAsync(Ae, Ae_d, sizeof(double) * nconfig * KN, cudaMemcpyDeviceToHost, ctx->stream));
    else memset(Ae, 0, sizeof(double) * nconfig * KN);
  }
  if (Af && n) IPG_RET(ipg_copy_d2h(ctx, Af, Af_d, sizeof(double) * 3 * n * KN));
  if (Aw) {
    if (n) CUDA_RET(ctx, cudaMemcpyAsync(Aw, Aw_d, sizeof(double) * 6 * nconfig * KN, cudaMemcpyDeviceToHost, ctx->stream));
    else memset(Aw, 0, sizeof(double) * 6 * nconfig * KN);
  }
  return ipg_status_check(ctx, "ipg_snap_batch_descriptors");
}

int ipg_snap_energy_forces_dev(ipg_snap* s, int64_t n, const double* d_pos, const int32_t* d_species,
                               const double L[3], const double* beta, double beta0, int32_t mode, double* d_E,
                               double* d_F, double* d_W6) {
  IPG_RET(check_common(s, n, d_pos, d_species, L));
  ipg_ctx* ctx = s->ctx;
  if (mode != IPG_SNAP_PLAIN && mode != IPG_SNAP_ADJOINT) return ipg_fail(ctx, IPG_ERR_ARG, "bad mode");
  if (!beta) return ipg_fail(ctx, IPG_ERR_ARG, "null beta");
  CUDA_RET(ctx, cudaSetDevice(ctx->device));
  IPG_RET(ipg_status_reset(ctx));
  EvalOut o;
  o.E = d_E;
  o.F = d_F;
  o.W6 = d_W6;
  int64_t aoff[2] = {0, n};
  IPG_RET(snap_eval(s, n, d_pos, d_species, 1, aoff, L, beta, beta0,
                    mode == IPG_SNAP_ADJOINT ? MODE_ADJ : MODE_PLAIN, o));
  return ipg_status_check(ctx, "ipg_snap_energy_forces_dev");
}

int ipg_snap_energy_forces(ipg_snap* s, int64_t n, const double* pos, const int32_t* species, const double L[3],
                           const double* beta, double beta0, int32_t mode, double* E, double* F, double* W6) {
  IPG_RET(check_common(s, n, pos, species, L));
  ipg_ctx* ctx = s->ctx;
  if (mode != IPG_SNAP_PLAIN && mode != IPG_SNAP_ADJOINT) return ipg_fail(ctx, IPG_ERR_ARG, "bad mode");
  if (!beta) return ipg_fail(ctx, IPG_ERR_ARG, "null beta");
  CUDA_RET(ctx, cudaSetDevice(ctx->device));
  IPG_RET(check_host_inputs(s, n, pos, species));
  double* d_pos;
  int32_t* d_sp;
  IPG_RET(upload_inputs(s, n, pos, species, &d_pos, &d_sp));
  IPG_RET(ipg_status_reset(ctx));
  double* d_out;  // [E, W6(6), pad, F(3n)]
  IPG_RET(scratch(ctx, "snap_out_EF", 3 * (size_t)n + 8, &d_out));
  EvalOut o;
  o.E = d_out;
  o.W6 = d_out + 1;
  o.F = F ? d_out + 8 : nullptr;
  int64_t aoff[2] = {0, n};
  IPG_RET(snap_eval(s, n, d_pos, d_sp, 1, aoff, L, beta, beta0, mode == IPG_SNAP_ADJOINT ? MODE_ADJ : MODE_PLAIN,
                    o));
  double head[8];
  CUDA_RET(ctx, cudaMemcpyAsync(head, d_out, sizeof(double) * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (F && n) IPG_RET(ipg_copy_d2h(ctx, F, d_out + 8, sizeof(double) * 3 * n));
  IPG_RET(ipg_status_check(ctx, "ipg_snap_energy_forces"));
  if (E) *E = head[0];
  if (W6) memcpy(W6, head + 1, 6 * sizeof(double));
  return IPG_OK;
}

}  // extern "C"

// Entry points that need the VJP kernel and batching live below, sharing the helpers.
namespace {

// gbeta = sum over blocks of the VJP partials (device), for device inputs already
// resident.  g = cotangent of forces [3n] (device), gE scalar.
// reuse_pl / reuse_utot: the pair list and Utot of an evaluation of the same positions just
// before (snap_eval's pl_out / utot_out), or null to build them here.
// reuse_Z: Z [idxz_max][n] of the same positions (k_snap_yrows<YM_YZ>), or null to form it here.
// v_out (optional): receives V [u_half][n] (V = sum_j (g_i - g_j) . d(sfac U_ij)/dr_ij) when the
// chain path formed it in one chunk, else null.
int snap_vjp_device(ipg_snap* s, int64_t n, const double* d_pos, const int32_t* d_species, int nconf,
                    const int64_t* h_atom_off, const double* h_L, const double* beta, double gE, const double* d_g,
                    double* d_gbeta, const PairList* reuse_pl, const double2* reuse_utot, const double2* reuse_Z,
                    const double2** v_out) {
  if (v_out) *v_out = nullptr;
  ipg_ctx* ctx = s->ctx;
  SnapDev dev = s->dev;
  if (dev.chem || dev.quadratic) {
    // element-resolved / quadratic SNAP: B and dB of every atom (compute_all_descriptors'
    // layouts), then gbeta[s][q] = gE sum_{i in s} B_i[q] + sum_a g_a . dB_a[s K + q]
    const int K = dev.K, nsp = dev.nsp;
    double *Bx, *dBx, *part;
    IPG_RET(scratch(ctx, "vjp_Bx", (size_t)n * K + 1, &Bx));
    IPG_RET(scratch(ctx, "vjp_dBx", (size_t)n * K * nsp * 3 + 1, &dBx));
    EvalOut o;
    o.B = Bx;
    o.dB = dBx;
    IPG_RET(snap_eval(s, n, d_pos, d_species, nconf, h_atom_off, h_L, beta, 0.0, MODE_DESC, o));
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>((n + 63) / 64, 1024));
    IPG_RET(scratch(ctx, "vjp_gpart", (size_t)grid * nsp * K + 1, &part));
    IPG_LAUNCH(ctx, k_gbeta_desc, (unsigned)grid, 128, 0, n, K, nsp, d_species, Bx, dBx, d_g, gE, part);
    IPG_LAUNCH(ctx, k_sum_partials, nblk((int64_t)nsp * K, 128), 128, 0, grid, nsp * K, part, d_gbeta, 0.0);
    return IPG_OK;
  }
  IPG_RET(set_beta(s, beta, 0.0, dev));
  PairList pl;
  if (reuse_pl)
    pl = *reuse_pl;
  else
    IPG_RET(snap_neighbors(s, n, d_pos, d_species, nconf, h_atom_off, h_L, pl));
  const int K = dev.K, nsp = dev.nsp;
  double* Ei;
  IPG_RET(scratch(ctx, "snap_Ei", (size_t)n + 1, &Ei));
  SnapIO io;
  memset(&io, 0, sizeof(io));
  io.n = n;
  io.off = pl.d_off;
  io.nbr = pl.d_j;
  io.rij = pl.d_r;
  io.species = d_species;
  io.Ei = Ei;
  io.g = d_g;
  io.gE = gE;
  io.status = ctx->d_status;
  if (reuse_pl && reuse_utot) {
    io.utot_in = reuse_utot;
  } else if (dev.J <= PAIR_CHAIN_MAX_J && !s->generic_adjoint && n) {
    double2* utot;
    IPG_RET(scratch(ctx, "snap_utot", (size_t)n * dev.idxu_max + 1, &utot));
    IPG_RET(launch_utot(ctx, dev, n, pl.d_off, pl.d_j, pl.d_r, d_species, utot, s->utot_warps, !s->utot_split));
    io.utot_in = utot;
  }
  if (io.utot_in && dev.J <= YR_MAX_J && s->h.yconst_ok) {
    // register-chain path: Z (row-blocked kernel) and V per chunk of atoms, then the
    // contraction
    const bool zgiven = reuse_Z && reuse_pl && reuse_utot;
    const int64_t C = zgiven ? n : zrows_chunk(s, dev, n);
    const int64_t nchunk = (n + C - 1) / C;
    double2 *Z, *V;
    if (zgiven)
      Z = const_cast<double2*>(reuse_Z);
    else
      IPG_RET(scratch(ctx, "snap_Z", (size_t)C * dev.idxz_max + 1, &Z));
    IPG_RET(scratch(ctx, "snap_vjp_V", (size_t)C * dev.u_half + 1, &V));
    int ysm, yper, gper = 1;
    IPG_RET(zrows_config(ctx, dev, &ysm, &yper));
    const bool withB = gE != 0.0;
    const int gsm = (int)((withB ? 2 : 1) * (size_t)dev.u_half * YS_ATOMS * sizeof(double2) + (size_t)nsp * K * 8);
    CUDA_RET(ctx, cudaFuncSetAttribute(k_snap_gbeta, cudaFuncAttributeMaxDynamicSharedMemorySize, gsm));
    CUDA_RET(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&gper, k_snap_gbeta, GB_WARPS * 32, gsm));
    const int64_t gmax = (int64_t)ctx->num_sms * std::max(1, gper);
    double* gpart;
    IPG_RET(scratch(ctx, "snap_gpart", (size_t)(nchunk * gmax) * nsp * K + 1, &gpart));
    int64_t rows = 0;  // partial rows written, in chunk order
    for (int64_t c = 0; c < nchunk; c++) {
      const int64_t a0 = c * C, nc = std::min(C, n - a0);
      const int64_t tiles = (nc + YS_ATOMS - 1) / YS_ATOMS;
      const int64_t yg = std::min<int64_t>(tiles, (int64_t)ctx->num_sms * std::max(1, yper));
      if (!zgiven)
        IPG_TIMED_LAUNCH(ctx, "snap_zrows", k_snap_yrows<YM_Z>, (unsigned)yg, YS_WARPS * 32, ysm, dev, s->h.yconst,
                         nc, d_species + a0, io.utot_in + (size_t)a0 * dev.idxu_max, Z, (double*)nullptr,
                         (double2*)nullptr);
      IPG_RET(launch_vsum(ctx, dev, a0, nc, pl.d_off, pl.d_j, pl.d_r, d_species, d_g, V, s->pair_tangent));
      const int64_t gg = std::min(tiles, gmax);
      IPG_TIMED_LAUNCH(ctx, "snap_gbeta", k_snap_gbeta, (unsigned)gg, GB_WARPS * 32, gsm, dev, a0, nc, d_species, Z,
                       V, io.utot_in, gE, gpart + (size_t)rows * nsp * K);
      rows += gg;
    }
    IPG_LAUNCH(ctx, k_sum_partials, nblk((int64_t)nsp * K, 128), 128, 0, rows, nsp * K, gpart, d_gbeta, 0.0);
    if (v_out && nchunk == 1) *v_out = V;
    return IPG_OK;
  }
  int threads = s->threads;
  SmemLayout L = smem_layout(dev, threads / 32, MODE_VJP, true);
  int per_sm = 1;
  CUDA_RET(ctx, cudaFuncSetAttribute(k_snap_atom<MODE_VJP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total));
  CUDA_RET(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_snap_atom<MODE_VJP>, threads, L.total));
  int64_t grid = std::min<int64_t>(std::max<int64_t>(n, 1), (int64_t)ctx->num_sms * std::max(1, per_sm));
  double* gpart;
  IPG_RET(scratch(ctx, "snap_gpart", (size_t)grid * nsp * K, &gpart));
  io.gpart = gpart;
  if (n) {
    IPG_RET(launch_atoms<MODE_VJP>(s, dev, io, n, &grid));
    IPG_LAUNCH(ctx, k_sum_partials, nblk((int64_t)nsp * K, 128), 128, 0, grid, nsp * K, gpart, d_gbeta, 0.0);
  } else {
    CUDA_RET(ctx, cudaMemsetAsync(d_gbeta, 0, sizeof(double) * nsp * K, ctx->stream));
  }
  return IPG_OK;
}

}  // namespace

extern "C" {

int ipg_snap_vjp_beta(ipg_snap* s, int64_t n, const double* pos, const int32_t* species, const double L[3], double gE,
                      const double* gF, double* gbeta, double* gbeta0) {
  IPG_RET(check_common(s, n, pos, species, L));
  ipg_ctx* ctx = s->ctx;
  if (!gbeta) return ipg_fail(ctx, IPG_ERR_ARG, "null gbeta");
  CUDA_RET(ctx, cudaSetDevice(ctx->device));
  IPG_RET(check_host_inputs(s, n, pos, species));
  double* d_pos;
  int32_t* d_sp;
  IPG_RET(upload_inputs(s, n, pos, species, &d_pos, &d_sp));
  IPG_RET(ipg_status_reset(ctx));
  const int K = s->dev.K, nsp = s->p.nspecies;
  double *d_g, *d_gb;
  IPG_RET(scratch(ctx, "snap_vjp_g", 3 * (size_t)n + 3, &d_g));
  IPG_RET(scratch(ctx, "snap_vjp_gb", (size_t)nsp * K, &d_gb));
  if (n) {
    if (gF) IPG_RET(ipg_copy_h2d(ctx, d_g, gF, sizeof(double) * 3 * n));
    else CUDA_RET(ctx, cudaMemsetAsync(d_g, 0, sizeof(double) * 3 * n, ctx->stream));
  }
  int64_t aoff[2] = {0, n};
  std::vector<double> zero_beta((size_t)nsp * K, 0.0);
  IPG_RET(snap_vjp_device(s, n, d_pos, d_sp, 1, aoff, L, zero_beta.data(), gE, d_g, d_gb, nullptr, nullptr, nullptr));
  CUDA_RET(ctx, cudaMemcpyAsync(gbeta, d_gb, sizeof(double) * nsp * K, cudaMemcpyDeviceToHost, ctx->stream));
  IPG_RET(ipg_status_check(ctx, "ipg_snap_vjp_beta"));
  if (gbeta0) *gbeta0 = gE;
  return IPG_OK;
}

int ipg_snap_vjp(ipg_snap* s, int64_t n, const double* pos, const int32_t* species, const double L[3],
                 const double* beta, double gE, const double* gF, double* gbeta, double* gbeta0, double* gpos) {
  IPG_RET(check_common(s, n, pos, species, L));
  ipg_ctx* ctx = s->ctx;
  if (gpos && !beta) return ipg_fail(ctx, IPG_ERR_ARG, "the position pullback needs beta");
  const SnapDev& d0 = s->dev;
  // both pullbacks from one evaluation: its list, Utot and Z (Y kernel in its Y+Z mode) serve
  // the beta pullback, whose V (gF contracted with dU/dr) is the Utot tangent of H gF
  const bool fused = gbeta && gpos && gF && n > 0 && !d0.chem && !d0.quadratic && d0.J <= YR_MAX_J &&
                     !s->generic_adjoint && !s->y_entries && s->h.yconst_ok && !s->generic_hvp;
  if (gbeta && !fused) IPG_RET(ipg_snap_vjp_beta(s, n, pos, species, L, gE, gF, gbeta, nullptr));
  if (gbeta0) *gbeta0 = gE;
  if (!gpos || n == 0) return IPG_OK;
  CUDA_RET(ctx, cudaSetDevice(ctx->device));
  IPG_RET(check_host_inputs(s, n, pos, species));
  if (gF && !host_all_finite(gF, 3 * n)) return ipg_fail(ctx, IPG_ERR_NONFINITE, "non-finite force cotangent");
  double* d_pos;
  int32_t* d_sp;
  IPG_RET(upload_inputs(s, n, pos, species, &d_pos, &d_sp));
  const size_t m = 3 * (size_t)n;
  double *F0, *Fd = nullptr, *gp;
  IPG_RET(scratch(ctx, "vjp_F0", m, &F0));
  IPG_RET(scratch(ctx, "vjp_gpos", m, &gp));
  IPG_RET(ipg_status_reset(ctx));
  int64_t aoff[2] = {0, n};
  EvalOut o;
  o.F = F0;
  PairList pl;
  o.pl_out = &pl;
  const double2 *utot = nullptr, *yw = nullptr, *Vg = nullptr;
  o.utot_out = &utot;
  o.yw_out = &yw;
  double2* Z = nullptr;
  bool zdone = false;
  double* d_gb = nullptr;
  if (fused) {
    IPG_RET(scratch(ctx, "vjp_Z", (size_t)d0.idxz_max * n + 1, &Z));
    IPG_RET(scratch(ctx, "snap_vjp_gb", (size_t)d0.nsp * d0.K, &d_gb));
    o.zall = Z;
    o.zall_done = &zdone;
  }
  IPG_RET(snap_eval(s, n, d_pos, d_sp, 1, aoff, L, beta, 0.0, MODE_ADJ, o));
  if (fused && !(zdone && utot && yw)) return ipg_fail(ctx, IPG_ERR_CUDA, "position pullback: evaluation without Z");
  if (gF) {
    // H gF: the tangent of the forces along gF, exact
    SnapDev dev = s->dev;
    if (dev.chem || dev.quadratic)
      return ipg_fail(ctx, IPG_ERR_UNSUPPORTED, "the position pullback of chem_flag / quadratic SNAP is not built");
    IPG_RET(set_beta(s, beta, 0.0, dev));
    double *d_v, *fd;
    IPG_RET(scratch(ctx, "vjp_v", m, &d_v));
    IPG_RET(scratch(ctx, "vjp_Fdot", m, &Fd));
    IPG_RET(scratch(ctx, "vjp_fdot", 3 * (size_t)pl.npairs + 3, &fd));
    IPG_RET(ipg_copy_h2d(ctx, d_v, gF, sizeof(double) * m));
    IPG_RET(ipg_side_join(ctx));
    if (fused) {
      IPG_RET(snap_vjp_device(s, n, d_pos, d_sp, 1, aoff, L, beta, gE, d_v, d_gb, &pl, utot, Z, &Vg));
      IPG_RET(set_beta(s, beta, 0.0, dev));
    }
    if (utot && yw && dev.J <= YR_MAX_J && !s->generic_hvp) {
      // register chains: Udot (k_snap_vsum), Ydot by polarization (two Y launches), the
      // second-order pair chains (k_snap_pair_hvp)
      const int U = dev.idxu_max, UH = dev.u_half;
      double2 *V, *Up, *Um, *Yp, *Ym, *Yd;
      double *sc, *ebuf;
      int32_t* owner;
      IPG_RET(scratch(ctx, "hvp_V", (size_t)UH * n + 1, &V));
      IPG_RET(scratch(ctx, "hvp_Up", (size_t)U * n + 1, &Up));
      IPG_RET(scratch(ctx, "hvp_Um", (size_t)U * n + 1, &Um));
      IPG_RET(scratch(ctx, "hvp_Yp", (size_t)UH * n + 1, &Yp));
      IPG_RET(scratch(ctx, "hvp_Ym", (size_t)UH * n + 1, &Ym));
      IPG_RET(scratch(ctx, "hvp_Yd", (size_t)UH * n + 1, &Yd));
      IPG_RET(scratch(ctx, "hvp_scale", (size_t)n, &sc));
      IPG_RET(scratch(ctx, "hvp_E", (size_t)n, &ebuf));
      IPG_RET(scratch(ctx, "snap_owner", (size_t)pl.npairs + 1, &owner));
      if (Vg)
        V = const_cast<double2*>(Vg);
      else
        IPG_RET(launch_vsum(ctx, dev, 0, n, pl.d_off, pl.d_j, pl.d_r, d_sp, d_v, V, s->pair_tangent));
      IPG_TIMED_LAUNCH(ctx, "snap_hvp", k_hvp_split, nblk(32 * n, 256), 256, 0, dev, n, utot, V, Up, Um, sc);
      bool d1 = false, d2 = false;
      IPG_RET(launch_y(s, dev, "snap_hvp_y", n, d_sp, Up, Yp, ebuf, nullptr, nullptr, &d1));
      IPG_RET(launch_y(s, dev, "snap_hvp_y", n, d_sp, Um, Ym, ebuf, nullptr, nullptr, &d2));
      if (!d1 || !d2) return ipg_fail(ctx, IPG_ERR_UNSUPPORTED, "position pullback: no atoms-in-lanes Y kernel");
      IPG_TIMED_LAUNCH(ctx, "snap_hvp", k_hvp_ydot, nblk((int64_t)UH * n, 256), 256, 0, n, UH, Yp, Ym, sc, Yd);
      IPG_LAUNCH(ctx, k_pair_owner, nblk(32 * n, 256), 256, 0, n, pl.d_off, owner);
      IPG_RET(launch_pair_hvp(ctx, dev, pl.npairs, pl.d_np, n, owner, pl.d_j, pl.d_r, d_sp, d_v, yw, Yd, fd,
                              s->pair_tangent));
    } else {
      // one block per atom, every phase in forward mode (k_snap_hvp)
      const int nw = 8;
      const HvpSmem HL = hvp_smem(dev, nw);
      if (HL.total > 227 * 1024)
        return ipg_fail(ctx, IPG_ERR_UNSUPPORTED,
                        "twojmax %d: the position pullback needs %zu bytes of shared memory", dev.J, HL.total);
      double* fv;
      IPG_RET(scratch(ctx, "vjp_fvec", 3 * (size_t)pl.npairs + 3, &fv));
      SnapIO io;
      memset(&io, 0, sizeof(io));
      io.n = n;
      io.off = pl.d_off;
      io.nbr = pl.d_j;
      io.rij = pl.d_r;
      io.species = d_sp;
      io.fvec = fv;
      io.status = ctx->d_status;
      CUDA_RET(ctx, cudaFuncSetAttribute(k_snap_hvp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HL.total));
      int per_sm = 1;
      CUDA_RET(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_snap_hvp, nw * 32, HL.total));
      const int64_t grid = std::min<int64_t>(n, (int64_t)ctx->num_sms * std::max(1, per_sm));
      IPG_TIMED_LAUNCH(ctx, "snap_hvp", k_snap_hvp, (unsigned)grid, nw * 32, HL.total, dev, io, d_v, fd);
    }
    IPG_LAUNCH(ctx, k_snap_gather, nblk(n, 128), 128, 0, n, pl.d_off, pl.d_j, pl.d_in_off, pl.d_in_pair, fd, 1,
               d_pos, Fd, (double*)nullptr);
  }
  IPG_LAUNCH(ctx, k_vjp_pos, nblk((int64_t)m, 256), 256, 0, (int64_t)m, F0, gE, Fd, gp);
  if (fused)
    CUDA_RET(ctx, cudaMemcpyAsync(gbeta, d_gb, sizeof(double) * d0.nsp * d0.K, cudaMemcpyDeviceToHost, ctx->stream));
  IPG_RET(ipg_copy_d2h(ctx, gpos, gp, sizeof(double) * m));
  return ipg_status_check(ctx, "ipg_snap_vjp");
}

int ipg_snap_autotune(ipg_snap* s, int64_t n, const double* pos, const int32_t* species, const double L[3],
                      const double* beta, const char* cache_path, char* report, int32_t report_len) {
  IPG_RET(check_common(s, n, pos, species, L));
  ipg_ctx* ctx = s->ctx;
  if (!beta) return ipg_fail(ctx, IPG_ERR_ARG, "null beta");
  CUDA_RET(ctx, cudaSetDevice(ctx->device));
  IPG_RET(check_host_inputs(s, n, pos, species));
  cudaDeviceProp prop;
  CUDA_RET(ctx, cudaGetDeviceProperties(&prop, ctx->device));
  int64_t cls = 1;
  while (cls < n) cls <<= 1;
  char kb[320];
  snprintf(kb, sizeof(kb), "%s|sm%d|twojmax%d|nsp%d|n%lld", prop.name, prop.multiProcessorCount, s->p.twojmax,
           s->p.nspecies, (long long)cls);
  const std::string key(kb);
  TuneChoice best;
  best.y_entries = s->y_entries;
  best.pair_split = s->pair_split;
  best.utot_split = s->utot_split;
  best.utot_warps = s->utot_warps;
  best.walk_warps = s->walk_warps;
  bool cached = cache_path && cache_path[0] && tune_cache_lookup(cache_path, key, best);
  int tried = 0;
  if (!cached && n > 0) {
    double* d_pos;
    int32_t* d_sp;
    IPG_RET(upload_inputs(s, n, pos, species, &d_pos, &d_sp));
    double *dE, *dF;
    IPG_RET(scratch(ctx, "tune_E", 1, &dE));
    IPG_RET(scratch(ctx, "tune_F", 3 * (size_t)n, &dF));
    cudaEvent_t e0, e1;
    CUDA_RET(ctx, cudaEventCreate(&e0));
    CUDA_RET(ctx, cudaEventCreate(&e1));
    int64_t aoff[2] = {0, n};
    EvalOut o;
    o.E = dE;
    o.F = dF;
    // best of 3 timed adjoint evaluations after one warm-up
    auto measure = [&](const TuneChoice& c, double* ms) -> int {
      tune_apply(s, c);
      IPG_RET(ipg_status_reset(ctx));
      IPG_RET(snap_eval(s, n, d_pos, d_sp, 1, aoff, L, beta, 0.0, MODE_ADJ, o));
      IPG_RET(ipg_status_check(ctx, "ipg_snap_autotune"));
      double b = 1e30;
      for (int r = 0; r < 3; r++) {
        CUDA_RET(ctx, cudaEventRecord(e0, ctx->stream));
        IPG_RET(snap_eval(s, n, d_pos, d_sp, 1, aoff, L, beta, 0.0, MODE_ADJ, o));
        CUDA_RET(ctx, cudaEventRecord(e1, ctx->stream));
        CUDA_RET(ctx, cudaEventSynchronize(e1));
        float t = 0.0f;
        CUDA_RET(ctx, cudaEventElapsedTime(&t, e0, e1));
        b = std::min(b, (double)t);
      }
      tried++;
      *ms = b;
      return IPG_OK;
    };
    int st = measure(best, &best.ms);
    // coordinate descent: each knob in turn, the others at their best so far
    const bool rows_ok = s->dev.J <= YR_MAX_J && s->h.yconst_ok, chains_ok = s->dev.J <= PAIR_CHAIN_MAX_J && !s->generic_adjoint;
    for (int knob = 0; knob < 5 && st == IPG_OK; knob++) {
      std::vector<int> vals;
      if (knob == 0 && rows_ok) vals = {0, 1};
      if (knob == 1 && chains_ok) vals = {0, 1};
      if (knob == 2 && chains_ok) vals = {0, 1};
      if (knob == 3 && chains_ok && best.utot_split) vals = {1, 2, 4};  // per-chain Utot kernels only
      if (knob == 4) vals = {1, 2, 4};
      for (int v : vals) {
        TuneChoice c = best;
        int* f = knob == 0 ? &c.y_entries : knob == 1 ? &c.pair_split : knob == 2 ? &c.utot_split
               : knob == 3 ? &c.utot_warps : &c.walk_warps;
        if (*f == v) continue;
        *f = v;
        st = measure(c, &c.ms);
        if (st) break;
        if (c.ms < best.ms) best = c;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) {
      tune_apply(s, TuneChoice());
      return st;
    }
    if (cache_path && cache_path[0]) {
      if (FILE* f = fopen(cache_path, "a")) {
        fprintf(f, "%s\n", tune_json(key, best, false, tried).c_str());
        fclose(f);
      }
    }
  }
  tune_apply(s, best);
  if (report && report_len > 0) {
    const std::string js = tune_json(key, best, cached, tried);
    snprintf(report, (size_t)report_len, "%s", js.c_str());
  }
  return IPG_OK;
}

int ipg_snap_batch_energy_forces_dev(ipg_snap* s, int32_t nconfig, const int64_t* atom_offsets, const double* d_pos,
                                     const int32_t* d_species, const double* L, const double* beta, double beta0,
                                     int32_t mode, int32_t graph, double* d_E, double* d_F, double* d_W6) {
  if (!s || nconfig < 1 || !atom_offsets || !L || !beta) return s ? ipg_fail(s->ctx, IPG_ERR_ARG, "bad batch args") : IPG_ERR_ARG;
  ipg_ctx* ctx = s->ctx;
  if (mode != IPG_SNAP_PLAIN && mode != IPG_SNAP_ADJOINT) return ipg_fail(ctx, IPG_ERR_ARG, "bad mode");
  if (atom_offsets[0] != 0) return ipg_fail(ctx, IPG_ERR_ARG, "atom_offsets[0] must be 0");
  for (int c = 0; c < nconfig; c++)
    if (atom_offsets[c + 1] < atom_offsets[c]) return ipg_fail(ctx, IPG_ERR_ARG, "atom_offsets must be non-decreasing");
  int64_t n = atom_offsets[nconfig];
  CUDA_RET(ctx, cudaSetDevice(ctx->device));
  EvalOut o;
  o.E = d_E;
  o.F = d_F;
  o.W6 = d_W6;
  const int emode = mode == IPG_SNAP_ADJOINT ? MODE_ADJ : MODE_PLAIN;
  bool periodic = true;
  for (int k = 0; k < 3 * nconfig; k++) periodic &= std::isfinite(L[k]);
  const bool use_graph = graph != 0 && periodic && n > 0;
  if (use_graph) {
    int st = batch_graph_replay(s, nconfig, atom_offsets, d_pos, d_species, L, beta, beta0, emode, o);
    if (st != IPG_ERR_CAPACITY && st != IPG_ERR_NOT_CAPTURED) return st;
  }
  IPG_RET(ipg_status_reset(ctx));
  IPG_RET(snap_eval(s, n, d_pos, d_species, nconfig, atom_offsets, L, beta, beta0, emode, o));
  IPG_RET(ipg_status_check(ctx, "ipg_snap_batch_energy_forces_dev"));
  if (use_graph) batch_graph_capture(s, nconfig, atom_offsets, d_pos, d_species, L, beta, beta0, emode, o);
  return IPG_OK;
}

int ipg_snap_batch_energy_forces(ipg_snap* s, int32_t nconfig, const int64_t* atom_offsets, const double* pos,
                                 const int32_t* species, const double* L, const double* beta, double beta0,
                                 int32_t mode, double* E, double* F, double* W6) {
  if (!s || nconfig < 1 || !atom_offsets || !L || !beta) return s ? ipg_fail(s->ctx, IPG_ERR_ARG, "bad batch args") : IPG_ERR_ARG;
  ipg_ctx* ctx = s->ctx;
  if (atom_offsets[0] != 0) return ipg_fail(ctx, IPG_ERR_ARG, "atom_offsets[0] must be 0");
  for (int c = 0; c < nconfig; c++)
    if (atom_offsets[c + 1] < atom_offsets[c]) return ipg_fail(ctx, IPG_ERR_ARG, "atom_offsets must be non-decreasing");
  int64_t n = atom_offsets[nconfig];
  IPG_RET(check_common(s, n, pos, species, L));
  CUDA_RET(ctx, cudaSetDevice(ctx->device));
  IPG_RET(check_host_inputs(s, n, pos, species));
  double* d_pos;
  int32_t* d_sp;
  IPG_RET(upload_inputs(s, n, pos, species, &d_pos, &d_sp));
  double* d_out;  // [E(nconf), W6(6 nconf), F(3n)]
  IPG_RET(scratch(ctx, "snap_out_batch", 7 * (size_t)nconfig + 3 * (size_t)n + 2, &d_out));
  IPG_RET(ipg_status_reset(ctx));
  EvalOut o;
  o.E = d_out;
  o.W6 = d_out + nconfig;
  o.F = F ? d_out + 7 * nconfig : nullptr;
  IPG_RET(snap_eval(s, n, d_pos, d_sp, nconfig, atom_offsets, L, beta, beta0,
                    mode == IPG_SNAP_ADJOINT ? MODE_ADJ : MODE_PLAIN, o));
  if (E) CUDA_RET(ctx, cudaMemcpyAsync(E, d_out, sizeof(double) * nconfig, cudaMemcpyDeviceToHost, ctx->stream));
  if (W6) CUDA_RET(ctx, cudaMemcpyAsync(W6, d_out + nconfig, sizeof(double) * 6 * nconfig, cudaMemcpyDeviceToHost, ctx->stream));
  if (F && n) IPG_RET(ipg_copy_d2h(ctx, F, d_out + 7 * nconfig, sizeof(double) * 3 * n));
  return ipg_status_check(ctx, "ipg_snap_batch_energy_forces");
}

int ipg_snap_batch_loss_grad(ipg_snap* s, int32_t nconfig, const int64_t* atom_offsets, const double* pos,
                             const int32_t* species, const double* L, const double* beta, double beta0,
                             const double* F_ref, double* loss, double* gbeta) {
  if (!s || nconfig < 1 || !atom_offsets || !L || !beta || !F_ref || !loss || !gbeta)
    return s ? ipg_fail(s->ctx, IPG_ERR_ARG, "bad batch args") : IPG_ERR_ARG;
  ipg_ctx* ctx = s->ctx;
  IPG_RET(check_offsets(ctx, nconfig, atom_offsets));
  int64_t n = atom_offsets[nconfig];
  IPG_RET(check_common(s, n, pos, species, L));
  CUDA_RET(ctx, cudaSetDevice(ctx->device));
  IPG_RET(check_host_inputs(s, n, pos, species));
  double* d_pos;
  int32_t* d_sp;
  IPG_RET(upload_inputs(s, n, pos, species, &d_pos, &d_sp));
  const int K = s->dev.K, nsp = s->p.nspecies;
  double *d_F, *d_Fref, *d_gb, *d_l;
  IPG_RET(scratch(ctx, "loss_F", 3 * (size_t)n + 3, &d_F));
  IPG_RET(scratch(ctx, "loss_Fref", 3 * (size_t)n + 3, &d_Fref));
  IPG_RET(scratch(ctx, "loss_gb", (size_t)nsp * K, &d_gb));
  IPG_RET(scratch(ctx, "loss_l", 1, &d_l));
  if (n) IPG_RET(ipg_copy_h2d(ctx, d_Fref, F_ref, sizeof(double) * 3 * n));
  IPG_RET(ipg_status_reset(ctx));
  EvalOut o;
  o.F = d_F;
  IPG_RET(snap_train_step(s, n, d_pos, d_sp, nconfig, atom_offsets, L, beta, beta0, d_Fref, o, d_l, d_gb, 0));
  CUDA_RET(ctx, cudaMemcpyAsync(gbeta, d_gb, sizeof(double) * nsp * K, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_RET(ctx, cudaMemcpyAsync(loss, d_l, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  return ipg_status_check(ctx, "ipg_snap_batch_loss_grad");
}

int ipg_snap_batch_loss_grad_dev(ipg_snap* s, int32_t nconfig, const int64_t* atom_offsets, const double* d_pos,
                                 const int32_t* d_species, const double* L, const double* beta, double beta0,
                                 const double* d_Fref, int32_t graph, double* d_E, double* d_F, double* d_W6,
                                 double* d_loss, double* d_gbeta) {
  if (!s || nconfig < 1 || !atom_offsets || !L || !beta || !d_Fref || !d_F || !d_loss || !d_gbeta)
    return s ? ipg_fail(s->ctx, IPG_ERR_ARG, "bad batch args") : IPG_ERR_ARG;
  ipg_ctx* ctx = s->ctx;
  IPG_RET(check_offsets(ctx, nconfig, atom_offsets));
  const int64_t n = atom_offsets[nconfig];
  if (n > 0 && (!d_pos || !d_species)) return ipg_fail(ctx, IPG_ERR_ARG, "null positions or species");
  CUDA_RET(ctx, cudaSetDevice(ctx->device));
  EvalOut o;
  o.E = d_E;
  o.F = d_F;
  o.W6 = d_W6;
  TrainBufs tb;
  tb.Fref = d_Fref;
  tb.loss = d_loss;
  tb.gbeta = d_gbeta;
  bool periodic = true;
  for (int k = 0; k < 3 * nconfig; k++) periodic &= std::isfinite(L[k]);
  const bool use_graph = graph != 0 && periodic && n > 0;
  if (use_graph) {
    int st = batch_graph_replay(s, nconfig, atom_offsets, d_pos, d_species, L, beta, beta0, MODE_TRAIN, o, tb);
    if (st != IPG_ERR_CAPACITY && st != IPG_ERR_NOT_CAPTURED) return st;
  }
  IPG_RET(ipg_status_reset(ctx));
  IPG_RET(snap_train_step(s, n, d_pos, d_species, nconfig, atom_offsets, L, beta, beta0, d_Fref, o, d_loss, d_gbeta,
                          0));
  IPG_RET(ipg_status_check(ctx, "ipg_snap_batch_loss_grad_dev"));
  if (use_graph) batch_graph_capture(s, nconfig, atom_offsets, d_pos, d_species, L, beta, beta0, MODE_TRAIN, o, tb);
  return IPG_OK;
}

}  // extern "C"
