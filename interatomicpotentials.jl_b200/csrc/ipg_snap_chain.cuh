// ipg_snap_chain.cuh — per-neighbor Wigner U / dU recursion held in registers.
//
// The recursion of compute_uarray / compute_duarray (compute_ui.jl:50-129, 186-326)
// builds row mb of level j from row mb of level j-1 only:
//   u_j[ma][mb] = rootpq[j-ma][j-mb] conj(a) u_{j-1}[ma][mb]
//               - rootpq[ma][j-mb]   conj(b) u_{j-1}[ma-1][mb]
// (and its derivative with respect to r_ij).  So the half plane (mb <= j/2) splits into
// J/2+1 independent "chains", chain mb being row mb of levels 2mb..J.  Chain mb starts
// from row mb of level 2mb-1, which is the inversion-symmetric mirror of row mb-1 of
// that level (compute_ui.jl:105-125): u[R][c] = (-1)^(c+R) conj(u[j-R][j-c]).  A thread
// therefore computes one chain of one neighbor entirely in registers: a short
// "staircase" (chain k over levels 2k+1, 2k+2 for k < mb) reaches the chain's start,
// then the chain runs to level J.  With twojmax a template parameter every index is a
// compile-time constant: no shared memory, no integer division, no divergence.
//
// The adjoint contraction (design of compute_dij.jl:5-74) is folded into the chain:
//   dE_i/dr_ij[k] = 2 sum_e w_e Re(conj(dsfac u_e uhat_k + sfac du_e[k]) Y_e)
//                 = 2 (dsfac uhat_k S0 + sfac S_k),
//   S0 = sum_e Re(conj(u_e) Yw_e),  S_k = sum_e Re(conj(du_e[k]) Yw_e),
// where Yw = w Y carries the half-plane weights (1, 1/2 on the middle element of even
// levels, 0 beyond it).
#pragma once

#include "ipg_snap.cuh"

namespace snapchain {

constexpr int RPQ_STRIDE = SNAP_MAX_J + 2;
// rootpq[p][q] = sqrt(p/q) (prebuilt_arrays.jl:314-321), one table for every twojmax.
__constant__ double c_rpq[RPQ_STRIDE * RPQ_STRIDE];

constexpr int half_block(int j) { return j <= 0 ? 0 : half_block(j - 1) + ((j - 1) / 2 + 1) * j; }

template <int J>
struct Chain {
  double2 u[J + 1];
  double2 d[3][J + 1];
};

struct Geom {
  double2 a, b;
  double2 da[3], db[3];
  double sfac, dsu[3];  // dsu[k] = dsfac * uhat_k
};

__device__ __forceinline__ double2 conjmul(double2 a, double2 v) {  // conj(a) * v
  return make_double2(a.x * v.x + a.y * v.y, a.x * v.y - a.y * v.x);
}

// Row mb: level j-1 -> level j, in place (descending ma keeps the old values needed).
template <int J, int j, int mb>
__device__ __forceinline__ void advance(Chain<J>& s, const Geom& G) {
#pragma unroll
  for (int ma = j; ma >= 0; --ma) {
    double2 nu = make_double2(0.0, 0.0);
    double2 nd[3];
#pragma unroll
    for (int k = 0; k < 3; k++) nd[k] = make_double2(0.0, 0.0);
    if (ma > 0) {
      const double rp = c_rpq[ma * RPQ_STRIDE + (j - mb)];
      const double2 v = s.u[ma - 1];
      const double2 t = conjmul(G.b, v);
      nu.x = -rp * t.x;
      nu.y = -rp * t.y;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const double2 t1 = conjmul(G.db[k], v);
        const double2 t2 = conjmul(G.b, s.d[k][ma - 1]);
        nd[k].x = -rp * (t1.x + t2.x);
        nd[k].y = -rp * (t1.y + t2.y);
      }
    }
    if (ma < j) {
      const double rp = c_rpq[(j - ma) * RPQ_STRIDE + (j - mb)];
      const double2 v = s.u[ma];
      const double2 t = conjmul(G.a, v);
      nu.x += rp * t.x;
      nu.y += rp * t.y;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const double2 t1 = conjmul(G.da[k], v);
        const double2 t2 = conjmul(G.a, s.d[k][ma]);
        nd[k].x += rp * (t1.x + t2.x);
        nd[k].y += rp * (t1.y + t2.y);
      }
    }
    s.u[ma] = nu;
#pragma unroll
    for (int k = 0; k < 3; k++) s.d[k][ma] = nd[k];
  }
}

// Row (j+1)/2 of an odd level from row (j-1)/2 by inversion symmetry.
template <int J, int j>
__device__ __forceinline__ void mirror(Chain<J>& s) {
  constexpr int R = (j + 1) / 2;
  double2 tu[j + 1];
  double2 td[3][j + 1];
#pragma unroll
  for (int c = 0; c <= j; c++) {
    tu[c] = s.u[j - c];
#pragma unroll
    for (int k = 0; k < 3; k++) td[k][c] = s.d[k][j - c];
  }
#pragma unroll
  for (int c = 0; c <= j; c++) {
    const double sg = ((c + R) & 1) ? -1.0 : 1.0;
    s.u[c] = make_double2(sg * tu[c].x, -sg * tu[c].y);
#pragma unroll
    for (int k = 0; k < 3; k++) s.d[k][c] = make_double2(sg * td[k][c].x, -sg * td[k][c].y);
  }
}

// Staircase: chain k from level 2k to 2k+1, mirror, chain k+1 to level 2k+2.
template <int J, int k, int MB>
__device__ __forceinline__ void staircase(Chain<J>& s, const Geom& G) {
  if constexpr (k < MB) {
    advance<J, 2 * k + 1, k>(s, G);
    mirror<J, 2 * k + 1>(s);
    advance<J, 2 * k + 2, k + 1>(s, G);
    staircase<J, k + 1, MB>(s, G);
  }
}

// Yw points at this atom's entry of h = 0 in the [h][atom] array; ys is the h stride.
template <int J, int j, int mb>
__device__ __forceinline__ void contract(const Chain<J>& s, const double2* __restrict__ Yw, int64_t ys, double& S0,
                                         double* S) {
  constexpr int base = half_block(j) + mb * (j + 1);
  constexpr int last = (2 * mb == j) ? mb : j;  // middle row of an even level stops at ma = j/2
#pragma unroll
  for (int ma = 0; ma <= last; ma++) {
    const double2 y = Yw[(base + ma) * ys];
    S0 += s.u[ma].x * y.x + s.u[ma].y * y.y;
#pragma unroll
    for (int k = 0; k < 3; k++) S[k] += s.d[k][ma].x * y.x + s.d[k][ma].y * y.y;
  }
}

template <int J, int j, int MB>
__device__ __forceinline__ void run_levels(Chain<J>& s, const Geom& G, const double2* __restrict__ Yw, int64_t ys,
                                           double& S0, double* S) {
  if constexpr (j <= J) {
    advance<J, j, MB>(s, G);
    contract<J, j, MB>(s, Yw, ys, S0, S);
    run_levels<J, j + 1, MB>(s, G, Yw, ys, S0, S);
  }
}

// Chain MB of one neighbor: returns S0 and S[3].
template <int J, int MB>
__device__ __forceinline__ void chain_adjoint(const Geom& G, const double2* __restrict__ Yw, int64_t ys, double& S0,
                                              double* S) {
  Chain<J> s;
#pragma unroll
  for (int c = 0; c <= J; c++) {
    s.u[c] = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < 3; k++) s.d[k][c] = make_double2(0.0, 0.0);
  }
  s.u[0] = make_double2(1.0, 0.0);  // level 0
  staircase<J, 0, MB>(s, G);
  S0 = 0.0;
  S[0] = S[1] = S[2] = 0.0;
  contract<J, 2 * MB, MB>(s, Yw, ys, S0, S);
  run_levels<J, 2 * MB + 1, MB>(s, G, Yw, ys, S0, S);
}

}  // namespace snapchain

namespace snapchain {

// ---- U only (Utot accumulation) ------------------------------------------------------
template <int J>
struct ChainU {
  double2 u[J + 1];
};

template <int J, int j, int mb>
__device__ __forceinline__ void advance_u(ChainU<J>& s, double2 a, double2 b) {
#pragma unroll
  for (int ma = j; ma >= 0; --ma) {
    double2 nu = make_double2(0.0, 0.0);
    if (ma > 0) {
      const double rp = c_rpq[ma * RPQ_STRIDE + (j - mb)];
      const double2 t = conjmul(b, s.u[ma - 1]);
      nu.x = -rp * t.x;
      nu.y = -rp * t.y;
    }
    if (ma < j) {
      const double rp = c_rpq[(j - ma) * RPQ_STRIDE + (j - mb)];
      const double2 t = conjmul(a, s.u[ma]);
      nu.x += rp * t.x;
      nu.y += rp * t.y;
    }
    s.u[ma] = nu;
  }
}

template <int J, int j>
__device__ __forceinline__ void mirror_u(ChainU<J>& s) {
  constexpr int R = (j + 1) / 2;
  double2 tu[j + 1];
#pragma unroll
  for (int c = 0; c <= j; c++) tu[c] = s.u[j - c];
#pragma unroll
  for (int c = 0; c <= j; c++) {
    const double sg = ((c + R) & 1) ? -1.0 : 1.0;
    s.u[c] = make_double2(sg * tu[c].x, -sg * tu[c].y);
  }
}

template <int J, int k, int MB>
__device__ __forceinline__ void staircase_u(ChainU<J>& s, double2 a, double2 b) {
  if constexpr (k < MB) {
    advance_u<J, 2 * k + 1, k>(s, a, b);
    mirror_u<J, 2 * k + 1>(s);
    advance_u<J, 2 * k + 2, k + 1>(s, a, b);
    staircase_u<J, k + 1, MB>(s, a, b);
  }
}

// Adds the warp-wide sum of sw * row mb of level j into acc[half_block(j) + mb*(j+1) + ma]
// (lane 0 writes; the calling warp owns these entries).
template <int J, int j, int mb>
__device__ __forceinline__ void reduce_row(const ChainU<J>& s, double sw, double2* __restrict__ acc, int lane) {
  constexpr int base = half_block(j) + mb * (j + 1);
#pragma unroll
  for (int ma = 0; ma <= j; ma++) {
    double x = sw * s.u[ma].x, y = sw * s.u[ma].y;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      x += __shfl_xor_sync(0xffffffffu, x, o);
      y += __shfl_xor_sync(0xffffffffu, y, o);
    }
    if (lane == 0) {
      acc[base + ma].x += x;
      acc[base + ma].y += y;
    }
  }
}

template <int J, int j, int MB>
__device__ __forceinline__ void run_levels_u(ChainU<J>& s, double2 a, double2 b, double sw, double2* acc, int lane) {
  if constexpr (j <= J) {
    advance_u<J, j, MB>(s, a, b);
    reduce_row<J, j, MB>(s, sw, acc, lane);
    run_levels_u<J, j + 1, MB>(s, a, b, sw, acc, lane);
  }
}

// Chain MB of one neighbor per lane (sw = 0 on idle lanes), reduced over the warp.
template <int J, int MB>
__device__ __forceinline__ void chain_utot(double2 a, double2 b, double sw, double2* acc, int lane) {
  ChainU<J> s;
#pragma unroll
  for (int c = 0; c <= J; c++) s.u[c] = make_double2(0.0, 0.0);
  s.u[0] = make_double2(1.0, 0.0);
  staircase_u<J, 0, MB>(s, a, b);
  reduce_row<J, 2 * MB, MB>(s, sw, acc, lane);
  run_levels_u<J, 2 * MB + 1, MB>(s, a, b, sw, acc, lane);
}

template <int J, int MB>
__device__ __forceinline__ void chain_utot_dispatch(int mb, double2 a, double2 b, double sw, double2* acc, int lane) {
  if constexpr (MB <= J / 2) {
    if (mb == MB) chain_utot<J, MB>(a, b, sw, acc, lane);
    else chain_utot_dispatch<J, MB + 1>(mb, a, b, sw, acc, lane);
  }
}

}  // namespace snapchain

namespace snapchain {

constexpr int u_block(int j) { return j * (j + 1) * (2 * j + 1) / 6; }  // idxu_block[j]

// Writes the warp-wide sum of sw * (row mb of level j) into the full Utot matrix: the
// entry itself and its inversion-symmetric mirror (compute_ui.jl:105-125); wself on the
// diagonal at the first neighbor chunk (zero_uarraytot, compute_ui.jl:131-152), later
// chunks accumulate.  Only lane 0 writes; the warp owns this atom's row mb entries.
template <int J, int j, int mb>
__device__ __forceinline__ void emit_row(const ChainU<J>& s, double sw, double2* __restrict__ ut, int lane,
                                         bool first, double wself) {
  constexpr int ub = u_block(j);
#pragma unroll
  for (int ma = 0; ma <= j; ma++) {
    if (2 * mb == j && ma > mb) continue;  // middle row: these are mirrors of ma' = j - ma
    double x = sw * s.u[ma].x, y = sw * s.u[ma].y;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      x += __shfl_xor_sync(0xffffffffu, x, o);
      y += __shfl_xor_sync(0xffffffffu, y, o);
    }
    if (lane == 0) {
      const int e = ub + mb * (j + 1) + ma;
      double2 v = first ? make_double2(ma == mb ? wself : 0.0, 0.0) : ut[e];
      v.x += x;
      v.y += y;
      ut[e] = v;
      if (!(2 * mb == j && ma == mb)) {
        const double sg = ((ma + mb) & 1) ? -1.0 : 1.0;
        ut[ub + (j - mb) * (j + 1) + (j - ma)] = make_double2(sg * v.x, -sg * v.y);
      }
    }
  }
}

template <int J, int j, int MB>
__device__ __forceinline__ void run_levels_emit(ChainU<J>& s, double2 a, double2 b, double sw, double2* ut,
                                                int lane, bool first, double wself) {
  if constexpr (j <= J) {
    advance_u<J, j, MB>(s, a, b);
    emit_row<J, j, MB>(s, sw, ut, lane, first, wself);
    run_levels_emit<J, j + 1, MB>(s, a, b, sw, ut, lane, first, wself);
  }
}

template <int J, int MB>
__device__ __forceinline__ void chain_utot_emit(double2 a, double2 b, double sw, double2* ut, int lane, bool first,
                                                double wself) {
  ChainU<J> s;
#pragma unroll
  for (int c = 0; c <= J; c++) s.u[c] = make_double2(0.0, 0.0);
  s.u[0] = make_double2(1.0, 0.0);
  staircase_u<J, 0, MB>(s, a, b);
  emit_row<J, 2 * MB, MB>(s, sw, ut, lane, first, wself);
  run_levels_emit<J, 2 * MB + 1, MB>(s, a, b, sw, ut, lane, first, wself);
}

}  // namespace snapchain

namespace snapchain {

// ---- all chains of one neighbor in one thread ------------------------------------------
// Chain mb's start row (row mb+1 of level 2mb+1, the mirror of chain mb's row there) is
// saved when chain mb passes that level and restored for chain mb+1: every half-plane
// entry is computed once, no staircase.  The saved row lives in shared memory as
// save[(comp * (J+1) + c) * nthreads + tid] (thread index fastest: conflict-free).
template <int J, int j>
__device__ __forceinline__ void save_mirror(const Chain<J>& s, double2* __restrict__ save, int nt, int tid) {
  constexpr int R = (j + 1) / 2;
#pragma unroll
  for (int c = 0; c <= j; c++) {
    const double sg = ((c + R) & 1) ? -1.0 : 1.0;
    const double2 u = s.u[j - c];
    save[(0 * (J + 1) + c) * nt + tid] = make_double2(sg * u.x, -sg * u.y);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const double2 d = s.d[k][j - c];
      save[((1 + k) * (J + 1) + c) * nt + tid] = make_double2(sg * d.x, -sg * d.y);
    }
  }
}

// The row mb is a runtime value: the level code exists once and each chain enters it at its start level (a switch
// that falls through the levels): the body of the kernel shrinks about (J/2+1)-fold, which
// the instruction cache needs at twojmax 8.  The rootpq factors come from constant memory
// by a uniform index; the recursion is written as FMA chains (rootpq scales a and its
// derivatives once per term, so each term costs 36 FP64 instructions instead of 42).
template <int J, int j>
__device__ __forceinline__ void advance_rt(Chain<J>& s, const Geom& G, int mb) {
  const int col = j - mb;
#pragma unroll
  for (int ma = j; ma >= 0; --ma) {
    double2 nu = make_double2(0.0, 0.0);
    double2 nd[3];
#pragma unroll
    for (int k = 0; k < 3; k++) nd[k] = make_double2(0.0, 0.0);
    if (ma > 0) {  // - rootpq[ma][j-mb] conj(b) u[ma-1]
      const double rp = -c_rpq[ma * RPQ_STRIDE + col];
      const double2 bb = make_double2(rp * G.b.x, rp * G.b.y);
      const double2 v = s.u[ma - 1];
      nu.x = fma(bb.x, v.x, bb.y * v.y);
      nu.y = fma(bb.x, v.y, -(bb.y * v.x));
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const double2 db = make_double2(rp * G.db[k].x, rp * G.db[k].y);
        const double2 dv = s.d[k][ma - 1];
        nd[k].x = fma(db.x, v.x, fma(db.y, v.y, fma(bb.x, dv.x, bb.y * dv.y)));
        nd[k].y = fma(db.x, v.y, fma(-db.y, v.x, fma(bb.x, dv.y, -(bb.y * dv.x))));
      }
    }
    if (ma < j) {  // + rootpq[j-ma][j-mb] conj(a) u[ma]
      const double rp = c_rpq[(j - ma) * RPQ_STRIDE + col];
      const double2 aa = make_double2(rp * G.a.x, rp * G.a.y);
      const double2 v = s.u[ma];
      nu.x = fma(aa.x, v.x, fma(aa.y, v.y, nu.x));
      nu.y = fma(aa.x, v.y, fma(-aa.y, v.x, nu.y));
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const double2 da = make_double2(rp * G.da[k].x, rp * G.da[k].y);
        const double2 dv = s.d[k][ma];
        nd[k].x = fma(da.x, v.x, fma(da.y, v.y, fma(aa.x, dv.x, fma(aa.y, dv.y, nd[k].x))));
        nd[k].y = fma(da.x, v.y, fma(-da.y, v.x, fma(aa.x, dv.y, fma(-aa.y, dv.x, nd[k].y))));
      }
    }
    s.u[ma] = nu;
#pragma unroll
    for (int k = 0; k < 3; k++) s.d[k][ma] = nd[k];
  }
}

template <int J, int j>
__device__ __forceinline__ void contract_rt(const Chain<J>& s, const double2* __restrict__ Yw, int64_t ys, int mb,
                                            double& S0, double* S) {
  const int last = (2 * mb == j) ? mb : j;  // middle row of an even level stops at ma = j/2
  const double2* y0 = Yw + (int64_t)(half_block(j) + mb * (j + 1)) * ys;
#pragma unroll
  for (int ma = 0; ma <= j; ma++) {
    if (ma > last) break;
    const double2 y = y0[ma * ys];
    S0 = fma(s.u[ma].x, y.x, fma(s.u[ma].y, y.y, S0));
#pragma unroll
    for (int k = 0; k < 3; k++) S[k] = fma(s.d[k][ma].x, y.x, fma(s.d[k][ma].y, y.y, S[k]));
  }
}

template <int J, int j>
__device__ __forceinline__ void level_rt(Chain<J>& s, const Geom& G, const double2* __restrict__ Yw, int64_t ys,
                                         int mb, double& S0, double* S, double2* save, int nt, int tid) {
  if constexpr (j <= J) {
    advance_rt<J, j>(s, G, mb);
    contract_rt<J, j>(s, Yw, ys, mb, S0, S);
    if constexpr (j % 2 == 1 && (j + 1) / 2 <= J / 2)
      if (j == 2 * mb + 1) save_mirror<J, j>(s, save, nt, tid);  // start row of chain mb+1
  }
}

template <int J>
__device__ __forceinline__ void load_row_rt(Chain<J>& s, const double2* __restrict__ save, int nt, int tid,
                                            int count) {
#pragma unroll
  for (int c = 0; c <= J; c++) {
    if (c >= count) break;
    s.u[c] = save[(0 * (J + 1) + c) * nt + tid];
#pragma unroll
    for (int k = 0; k < 3; k++) s.d[k][c] = save[((1 + k) * (J + 1) + c) * nt + tid];
  }
}

template <int J>
__device__ __forceinline__ void all_chains_adjoint(const Geom& G, const double2* __restrict__ Yw, int64_t ys,
                                                   double& S0, double* S, double2* save, int nt, int tid) {
  static_assert(J <= 12, "level switch covers twojmax <= 12");
  Chain<J> s;
#pragma unroll
  for (int c = 0; c <= J; c++) {
    s.u[c] = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < 3; k++) s.d[k][c] = make_double2(0.0, 0.0);
  }
  s.u[0] = make_double2(1.0, 0.0);
  S0 = 0.0;
  S[0] = S[1] = S[2] = 0.0;
  contract<J, 0, 0>(s, Yw, ys, S0, S);
#pragma unroll 1
  for (int mb = 0; mb <= J / 2; mb++) {
    if (mb > 0) {
      asm volatile("" ::: "memory");  // this chain's loads stay after the previous chain's saves
      load_row_rt<J>(s, save, nt, tid, 2 * mb);  // row mb of level 2mb-1
    }
    switch (mb == 0 ? 1 : 2 * mb) {  // chain mb runs levels 2mb (1 for chain 0) .. J
#define IPG_LEVEL(JJ) \
  case JJ:            \
    level_rt<J, JJ>(s, G, Yw, ys, mb, S0, S, save, nt, tid);
      IPG_LEVEL(1) IPG_LEVEL(2) IPG_LEVEL(3) IPG_LEVEL(4) IPG_LEVEL(5) IPG_LEVEL(6)
      IPG_LEVEL(7) IPG_LEVEL(8) IPG_LEVEL(9) IPG_LEVEL(10) IPG_LEVEL(11) IPG_LEVEL(12)
#undef IPG_LEVEL
      default:
        break;
    }
  }
}

}  // namespace snapchain

namespace snapchain {

// ---- Utot, all chains of a neighbor per lane, one launch ----------------------------------
// advance_u with the row mb a runtime value (FMA chains; rootpq scales a and b per term).
template <int J, int j>
__device__ __forceinline__ void advance_u_rt(ChainU<J>& s, double2 a, double2 b, int mb) {
  const int col = j - mb;
#pragma unroll
  for (int ma = j; ma >= 0; --ma) {
    double2 nu = make_double2(0.0, 0.0);
    if (ma > 0) {  // - rootpq[ma][j-mb] conj(b) u[ma-1]
      const double rp = -c_rpq[ma * RPQ_STRIDE + col];
      const double bx = rp * b.x, by = rp * b.y;
      const double2 v = s.u[ma - 1];
      nu.x = fma(bx, v.x, by * v.y);
      nu.y = fma(bx, v.y, -(by * v.x));
    }
    if (ma < j) {  // + rootpq[j-ma][j-mb] conj(a) u[ma]
      const double rp = c_rpq[(j - ma) * RPQ_STRIDE + col];
      const double ax = rp * a.x, ay = rp * a.y;
      const double2 v = s.u[ma];
      nu.x = fma(ax, v.x, fma(ay, v.y, nu.x));
      nu.y = fma(ax, v.y, fma(-ay, v.x, nu.y));
    }
    s.u[ma] = nu;
  }
}

// Warp-wide sums of staged elements.  Each lane (one neighbor) stages sw * U of up to
// UT_SLOTS elements in shared memory as buf[slot][lane] (33 columns: fewer bank conflicts);
// a flush has lane pair (2q, 2q+1) sum the real and imaginary part of slot q over the 32
// lanes in fixed order and write the Utot entry and its inversion-symmetric mirror.
constexpr int UT_SLOTS = 16;
static_assert(2 * UT_SLOTS <= 32, "a flush sums one slot per lane pair: at most 16 slots");
struct UtStage {
  double2* buf;  // [UT_SLOTS][33] of this warp
  int* dst;      // [UT_SLOTS] packed destination of each slot
  double* ut;    // this atom's entry 0, as doubles; entry e at ut[2 e stride + c]
  int64_t stride = 1;
  int lane, nslot;
  bool first;    // first chunk of neighbors: write (with wself on the diagonal), else add
  double wself;
  // packed destination: entry e | mirror e' << 12 | mirror sign << 24 | diagonal << 25 | has mirror << 26
  // stages one element; the caller makes room first (room(), once per row)
  __device__ __forceinline__ void push(double2 v, int packed) {
    buf[nslot * 33 + lane] = v;
    if (lane == 0) dst[nslot] = packed;
    ++nslot;
  }
  __device__ __forceinline__ void room(int need) {
    if (nslot + need > UT_SLOTS) flush();
  }
  __device__ __forceinline__ void flush() {
    __syncwarp();
    const int q = lane >> 1, c = lane & 1;
    if (q < nslot) {
      const double* col = reinterpret_cast<const double*>(buf + q * 33) + c;
      double t4[4] = {0.0, 0.0, 0.0, 0.0};  // four partial sums: a shorter dependency chain
#pragma unroll
      for (int k = 0; k < 32; k++) t4[k & 3] += col[2 * k];
      const double t = (t4[0] + t4[1]) + (t4[2] + t4[3]);
      const int pk = dst[q];
      const int e = pk & 0xfff;
      double* pe = ut + 2 * (int64_t)e * stride + c;
      double v = first ? ((c == 0 && ((pk >> 25) & 1)) ? wself : 0.0) : *pe;
      v += t;
      *pe = v;
      if ((pk >> 26) & 1) {
        const double sg = ((pk >> 24) & 1) ? -1.0 : 1.0;
        ut[2 * (int64_t)((pk >> 12) & 0xfff) * stride + c] = c ? -sg * v : sg * v;
      }
    }
    __syncwarp();
    nslot = 0;
  }
};

// Stages row mb of level j (the half-plane part) with its destinations in the full Utot.
// The chain carries sw U (the recursion is linear and sw real, so starting it from sw instead
// of 1 scales every entry, the mirrored rows included): the staged values need no multiply.
template <int J, int j>
__device__ __forceinline__ void stage_row(const ChainU<J>& s, int mb, UtStage& st) {
  static_assert(j + 1 <= UT_SLOTS, "a row must fit the staging buffer");
  const int last = (2 * mb == j) ? mb : j;  // middle row: entries beyond ma = mb are mirrors
  const int ub = u_block(j);
  st.room(last + 1);
#pragma unroll
  for (int ma = 0; ma <= j; ma++) {
    if (ma > last) break;
    const int e = ub + mb * (j + 1) + ma;
    const bool self_mirror = (2 * mb == j) && ma == mb;
    const int em = ub + (j - mb) * (j + 1) + (j - ma);
    const int packed = e | (em << 12) | (((ma + mb) & 1) << 24) | ((ma == mb) << 25) | ((!self_mirror) << 26);
    st.push(s.u[ma], packed);
  }
}

template <int J, int j>
__device__ __forceinline__ void level_u_rt(ChainU<J>& s, double2 a, double2 b, int mb, UtStage& st,
                                           double2 (&sv)[J + 1]) {
  if constexpr (j <= J) {
    advance_u_rt<J, j>(s, a, b, mb);
    stage_row<J, j>(s, mb, st);
    if constexpr (j % 2 == 1 && (j + 1) / 2 <= J / 2) {
      if (j == 2 * mb + 1) {  // start row of chain mb+1: the mirror of this row
        constexpr int R = (j + 1) / 2;
#pragma unroll
        for (int c = 0; c <= j; c++) {
          const double sg = ((c + R) & 1) ? -1.0 : 1.0;
          sv[c] = make_double2(sg * s.u[j - c].x, -sg * s.u[j - c].y);
        }
      }
    }
  }
}

// All chains of one neighbor (sw = 0 on idle lanes), every half-plane entry computed once.
template <int J>
__device__ __forceinline__ void all_chains_utot(double2 a, double2 b, double sw, UtStage& st) {
  static_assert(J <= 12, "level switch covers twojmax <= 12");
  ChainU<J> s;
  double2 sv[J + 1];
#pragma unroll
  for (int c = 0; c <= J; c++) {
    s.u[c] = make_double2(0.0, 0.0);
    sv[c] = make_double2(0.0, 0.0);
  }
  s.u[0] = make_double2(sw, 0.0);
  stage_row<J, 0>(s, 0, st);
#pragma unroll 1
  for (int mb = 0; mb <= J / 2; mb++) {
    if (mb > 0) {
#pragma unroll
      for (int c = 0; c <= J; c++)
        if (c < 2 * mb) s.u[c] = sv[c];
    }
    switch (mb == 0 ? 1 : 2 * mb) {  // chain mb runs levels 2mb (1 for chain 0) .. J
#define IPG_LEVEL(JJ) \
  case JJ:            \
    level_u_rt<J, JJ>(s, a, b, mb, st, sv);
      IPG_LEVEL(1) IPG_LEVEL(2) IPG_LEVEL(3) IPG_LEVEL(4) IPG_LEVEL(5) IPG_LEVEL(6)
      IPG_LEVEL(7) IPG_LEVEL(8) IPG_LEVEL(9) IPG_LEVEL(10) IPG_LEVEL(11) IPG_LEVEL(12)
#undef IPG_LEVEL
      default:
        break;
    }
  }
  st.flush();
}

// ---- adjoint forces from U alone (the SU(2) derivative identity) ------------------------
// U^j(r) is the spin-j/2 representation of the unit quaternion (a, b), g = [[conj a, -conj b],
// [b, a]] (the level-1 matrix of the recursion), so its derivative along r_k is U^j times
// the representation of the Lie-algebra element g^-1 dg/dr_k = [[i al_k, be_k], [-conj be_k,
// -i al_k]], acting on the column index ma:
//   dU/dr_k = U (al_k D1 + Re(be_k) D2 + Im(be_k) D3),
//   D1 = diag(i (j - 2 ma)),  D2[m][m+1] = s_m = -D2[m+1][m],  D3[m][m+1] = D3[m+1][m] = i s_m,
//   s_m = sqrt((m + 1)(j - m)),
//   al_k = Im(a conj(da_k) + conj(b) db_k),  be_k = conj(b) da_k - a conj(db_k).
// So the adjoint sums S_k = sum_e Re(conj(dU_e/dr_k) Yw_e) over the half plane are
//   S_k = al_k T1 + Re(be_k) T2 + Im(be_k) T3,
//   T1 = sum_e (j - 2 ma) Im(conj(U_e) Yw_e),  T2 = sum_e Re(conj(U_e) Y2_e),  T3 = sum_e Re(conj(U_e) Y3_e),
// with, within each row (Yw zero beyond a row's weighted entries),
//   Y2[m] = s_m Yw[m+1] - s_{m-1} Yw[m-1],  Y3[m] = -i (s_m Yw[m+1] + s_{m-1} Yw[m-1]),
// which depend on the centre atom only.  A pair then needs U alone, without the three
// tangent chains: about a quarter of the FP64 work of all_chains_adjoint, same result up to
// rounding.  y: the staged Yw, Y2, Y3 of the pair's atom, entry h of array g at
// y[(g ya + h) ys]; acc: S0, T1, T2, T3 for even ma, then for odd ma (shorter FMA chains).
template <int J, int j>
__device__ __forceinline__ void contract_lie(const ChainU<J>& s, const double2* __restrict__ y, int ys, int ya,
                                             int mb, double (&acc)[8]) {
  // the middle row of an even level: Yw ends at ma = mb, Y2 and Y3 one entry later
  const int lim = (2 * mb == j) ? (mb < j ? mb + 1 : j) : j;
  const double2* y0 = y + (half_block(j) + mb * (j + 1)) * ys;
#pragma unroll
  for (int ma = 0; ma <= j; ma++) {
    if (ma > lim) break;
    const int q = 4 * (ma & 1);  // a compile-time index once the loop is unrolled
    const double2 u = s.u[ma];
    const double2 w = y0[ma * ys], w2 = y0[(ya + ma) * ys], w3 = y0[(2 * ya + ma) * ys];
    acc[q] = fma(u.x, w.x, fma(u.y, w.y, acc[q]));
    if (j != 2 * ma) acc[q + 1] = fma((double)(j - 2 * ma), fma(u.x, w.y, -(u.y * w.x)), acc[q + 1]);
    acc[q + 2] = fma(u.x, w2.x, fma(u.y, w2.y, acc[q + 2]));
    acc[q + 3] = fma(u.x, w3.x, fma(u.y, w3.y, acc[q + 3]));
  }
}

template <int J, int j>
__device__ __forceinline__ void level_lie_rt(ChainU<J>& s, double2 a, double2 b, int mb, const double2* y, int ys,
                                             int ya, double (&acc)[8], double2 (&sv)[J + 1]) {
  if constexpr (j <= J) {
    advance_u_rt<J, j>(s, a, b, mb);
    contract_lie<J, j>(s, y, ys, ya, mb, acc);
    if constexpr (j % 2 == 1 && (j + 1) / 2 <= J / 2) {
      if (j == 2 * mb + 1) {  // start row of chain mb+1: the mirror of this row
        constexpr int R = (j + 1) / 2;
#pragma unroll
        for (int c = 0; c <= j; c++) {
          const double sg = ((c + R) & 1) ? -1.0 : 1.0;
          sv[c] = make_double2(sg * s.u[j - c].x, -sg * s.u[j - c].y);
        }
      }
    }
  }
}

// All chains of one neighbor, U only, contracted with the centre atom's Yw, Y2, Y3.
template <int J>
__device__ __forceinline__ void all_chains_lie(double2 a, double2 b, const double2* __restrict__ y, int ys, int ya,
                                               double& S0, double (&T)[3]) {
  static_assert(J <= 12, "level switch covers twojmax <= 12");
  ChainU<J> s;
  double2 sv[J + 1];
#pragma unroll
  for (int c = 0; c <= J; c++) {
    s.u[c] = make_double2(0.0, 0.0);
    sv[c] = make_double2(0.0, 0.0);
  }
  s.u[0] = make_double2(1.0, 0.0);
  double acc[8];
#pragma unroll
  for (int q = 0; q < 8; q++) acc[q] = 0.0;
  contract_lie<J, 0>(s, y, ys, ya, 0, acc);
#pragma unroll 1
  for (int mb = 0; mb <= J / 2; mb++) {
    if (mb > 0) {
#pragma unroll
      for (int c = 0; c <= J; c++)
        if (c < 2 * mb) s.u[c] = sv[c];
    }
    switch (mb == 0 ? 1 : 2 * mb) {  // chain mb runs levels 2mb (1 for chain 0) .. J
#define IPG_LEVEL(JJ) \
  case JJ:            \
    level_lie_rt<J, JJ>(s, a, b, mb, y, ys, ya, acc, sv);
      IPG_LEVEL(1) IPG_LEVEL(2) IPG_LEVEL(3) IPG_LEVEL(4) IPG_LEVEL(5) IPG_LEVEL(6)
      IPG_LEVEL(7) IPG_LEVEL(8) IPG_LEVEL(9) IPG_LEVEL(10) IPG_LEVEL(11) IPG_LEVEL(12)
#undef IPG_LEVEL
      default:
        break;
    }
  }
  S0 = acc[0] + acc[4];
#pragma unroll
  for (int g = 0; g < 3; g++) T[g] = acc[1 + g] + acc[5 + g];
}

}  // namespace snapchain

namespace snapchain {

// ---- V = sum over neighbors of g_ij . dU/dr_ij (the beta pullback of the forces) --------
// Per lane one neighbor, all chains with derivatives (the runtime-row level code of the
// adjoint kernel); each half-plane entry h contributes
//   v_h = sum_k gv_k (dsfac uhat_k u_h + sfac du_k,h) = A u_h + sum_k B_k du_k,h
// (A = dsfac gv.uhat, B_k = sfac gv_k), summed over the warp's lanes through the staging
// buffer into V[h] of the atom.
template <int J, int j>
__device__ __forceinline__ void stage_v(const Chain<J>& s, double A, const double* Bk, int mb, UtStage& st) {
  const int last = (2 * mb == j) ? mb : j;
  const int hb = half_block(j) + mb * (j + 1);
  st.room(last + 1);
#pragma unroll
  for (int ma = 0; ma <= j; ma++) {
    if (ma > last) break;
    double vx = A * s.u[ma].x, vy = A * s.u[ma].y;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      vx = fma(Bk[k], s.d[k][ma].x, vx);
      vy = fma(Bk[k], s.d[k][ma].y, vy);
    }
    st.push(make_double2(vx, vy), hb + ma);  // packed: entry only (no mirror, no diagonal)
  }
}

template <int J, int j>
__device__ __forceinline__ void level_v(Chain<J>& s, const Geom& G, double A, const double* Bk, int mb, UtStage& st,
                                        double2* save, int nt, int tid) {
  if constexpr (j <= J) {
    advance_rt<J, j>(s, G, mb);
    stage_v<J, j>(s, A, Bk, mb, st);
    if constexpr (j % 2 == 1 && (j + 1) / 2 <= J / 2)
      if (j == 2 * mb + 1) save_mirror<J, j>(s, save, nt, tid);
  }
}

template <int J>
__device__ __forceinline__ void all_chains_v(const Geom& G, double A, const double* Bk, UtStage& st, double2* save,
                                             int nt, int tid) {
  static_assert(J <= 12, "level switch covers twojmax <= 12");
  Chain<J> s;
#pragma unroll
  for (int c = 0; c <= J; c++) {
    s.u[c] = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < 3; k++) s.d[k][c] = make_double2(0.0, 0.0);
  }
  s.u[0] = make_double2(1.0, 0.0);
  stage_v<J, 0>(s, A, Bk, 0, st);
#pragma unroll 1
  for (int mb = 0; mb <= J / 2; mb++) {
    if (mb > 0) {
      asm volatile("" ::: "memory");
      load_row_rt<J>(s, save, nt, tid, 2 * mb);
    }
    switch (mb == 0 ? 1 : 2 * mb) {
#define IPG_LEVEL(JJ) \
  case JJ:            \
    level_v<J, JJ>(s, G, A, Bk, mb, st, save, nt, tid);
      IPG_LEVEL(1) IPG_LEVEL(2) IPG_LEVEL(3) IPG_LEVEL(4) IPG_LEVEL(5) IPG_LEVEL(6)
      IPG_LEVEL(7) IPG_LEVEL(8) IPG_LEVEL(9) IPG_LEVEL(10) IPG_LEVEL(11) IPG_LEVEL(12)
#undef IPG_LEVEL
      default:
        break;
    }
  }
  st.flush();
}

// ---- V from U alone (the generator identity of all_chains_lie) --------------------------
// sum_k B_k dU/dr_k = U (g1 D1 + g2 D2 + g3 D3) with g = sum_k B_k (al_k, Re be_k, Im be_k),
// so within a row (s_m = c_sgen[j][mb][m])
//   v[ma] = A u[ma] + g1 (j - 2 ma) i u[ma] + s_{ma-1} (g2 + i g3) u[ma-1] + s_ma (i g3 - g2) u[ma+1]:
// the same V as all_chains_v without the three tangent chains.
// [j][mb][m] = sqrt((m + 1)(j - m)), 0 <= m < j, the same for every row mb <= j/2: indexed by the
// runtime row so that the compiler loads the factors where they are used instead of hoisting
// all of them into registers for the whole neighbor loop (which spilled)
constexpr int SGEN_ROWS = SNAP_MAX_J / 2 + 1;
__constant__ double c_sgen[RPQ_STRIDE * SGEN_ROWS * RPQ_STRIDE];

template <int J, int j>
__device__ __forceinline__ void stage_vlie(const ChainU<J>& s, double A, double g1, double g2, double g3, int mb,
                                           UtStage& st) {
  const int last = (2 * mb == j) ? mb : j;
  const int hb = half_block(j) + mb * (j + 1);
  st.room(last + 1);
#pragma unroll
  for (int ma = 0; ma <= j; ma++) {
    if (ma > last) break;
    const double2 u = s.u[ma];
    const double c1 = g1 * (double)(j - 2 * ma);  // i u = (-u.y, u.x)
    double vx = fma(A, u.x, -(c1 * u.y)), vy = fma(A, u.y, c1 * u.x);
    if (ma > 0) {  // s_{ma-1} (g2 + i g3) u[ma-1]
      const double sg = c_sgen[(j * SGEN_ROWS + mb) * RPQ_STRIDE + ma - 1];
      const double2 w = s.u[ma - 1];
      const double px = sg * g2, py = sg * g3;
      vx = fma(px, w.x, fma(-py, w.y, vx));
      vy = fma(px, w.y, fma(py, w.x, vy));
    }
    if (ma < j) {  // s_ma (-g2 + i g3) u[ma+1]
      const double sg = c_sgen[(j * SGEN_ROWS + mb) * RPQ_STRIDE + ma];
      const double2 w = s.u[ma + 1];
      const double px = -sg * g2, py = sg * g3;
      vx = fma(px, w.x, fma(-py, w.y, vx));
      vy = fma(px, w.y, fma(py, w.x, vy));
    }
    st.push(make_double2(vx, vy), hb + ma);  // packed: entry only (no mirror, no diagonal)
  }
}

template <int J, int j>
__device__ __forceinline__ void level_vlie(ChainU<J>& s, double2 a, double2 b, double A, double g1, double g2,
                                           double g3, int mb, UtStage& st, double2 (&sv)[J + 1]) {
  if constexpr (j <= J) {
    advance_u_rt<J, j>(s, a, b, mb);
    stage_vlie<J, j>(s, A, g1, g2, g3, mb, st);
    if constexpr (j % 2 == 1 && (j + 1) / 2 <= J / 2) {
      if (j == 2 * mb + 1) {  // start row of chain mb+1: the mirror of this row
        constexpr int R = (j + 1) / 2;
#pragma unroll
        for (int c = 0; c <= j; c++) {
          const double sg = ((c + R) & 1) ? -1.0 : 1.0;
          sv[c] = make_double2(sg * s.u[j - c].x, -sg * s.u[j - c].y);
        }
      }
    }
  }
}

template <int J>
__device__ __forceinline__ void all_chains_vlie(double2 a, double2 b, double A, double g1, double g2, double g3,
                                                UtStage& st) {
  static_assert(J <= 12, "level switch covers twojmax <= 12");
  ChainU<J> s;
  double2 sv[J + 1];
#pragma unroll
  for (int c = 0; c <= J; c++) {
    s.u[c] = make_double2(0.0, 0.0);
    sv[c] = make_double2(0.0, 0.0);
  }
  s.u[0] = make_double2(1.0, 0.0);
  stage_vlie<J, 0>(s, A, g1, g2, g3, 0, st);
#pragma unroll 1
  for (int mb = 0; mb <= J / 2; mb++) {
    if (mb > 0) {
#pragma unroll
      for (int c = 0; c <= J; c++)
        if (c < 2 * mb) s.u[c] = sv[c];
    }
    switch (mb == 0 ? 1 : 2 * mb) {
#define IPG_LEVEL(JJ) \
  case JJ:            \
    level_vlie<J, JJ>(s, a, b, A, g1, g2, g3, mb, st, sv);
      IPG_LEVEL(1) IPG_LEVEL(2) IPG_LEVEL(3) IPG_LEVEL(4) IPG_LEVEL(5) IPG_LEVEL(6)
      IPG_LEVEL(7) IPG_LEVEL(8) IPG_LEVEL(9) IPG_LEVEL(10) IPG_LEVEL(11) IPG_LEVEL(12)
#undef IPG_LEVEL
      default:
        break;
    }
  }
  st.flush();
}

// ---- the Hessian-vector product of the pair forces from U and one tangent ---------------
// The pair force of all_chains_lie, F_k = c0_k S0 + sum_g cT_kg T_g, has along the pair
// displacement tangent rdot the tangent
//   Fdot_k = c0dot_k S0 + c0_k (S0a + S0b) + sum_g [cTdot_kg T_g + cT_kg (T_g,a + T_g,b)],
// where the a-terms contract the tangent Udot of U (one tangent chain along rdot) with Yw and
// the b-terms contract U with the centre atom's Ydot (Yd).  The generator rows U D_g are
// formed from the row of U in registers ((U D1)[m] = i (j - 2m) U[m], (U D2)[m] = s_{m-1}
// U[m-1] - s_m U[m+1], (U D3)[m] = i (s_{m-1} U[m-1] + s_m U[m+1])), so only Yw and Yd are
// read.  acc: S0, S0a, S0b, then T_g, T_g,a, T_g,b for g = 1, 2, 3.
template <int J>
struct ChainT {
  double2 u[J + 1];
  double2 t[J + 1];  // the tangent of u along rdot
};

template <int J, int j>
__device__ __forceinline__ void advance_t_rt(ChainT<J>& s, double2 a, double2 at, double2 b, double2 bt, int mb) {
  const int col = j - mb;
#pragma unroll
  for (int ma = j; ma >= 0; --ma) {
    double2 nu = make_double2(0.0, 0.0), nt = make_double2(0.0, 0.0);
    if (ma > 0) {  // - rootpq[ma][j-mb] conj(b) u[ma-1]
      const double rp = -c_rpq[ma * RPQ_STRIDE + col];
      const double bx = rp * b.x, by = rp * b.y, btx = rp * bt.x, bty = rp * bt.y;
      const double2 v = s.u[ma - 1], vt = s.t[ma - 1];
      nu.x = fma(bx, v.x, by * v.y);
      nu.y = fma(bx, v.y, -(by * v.x));
      nt.x = fma(btx, v.x, fma(bty, v.y, fma(bx, vt.x, by * vt.y)));
      nt.y = fma(btx, v.y, fma(-bty, v.x, fma(bx, vt.y, -(by * vt.x))));
    }
    if (ma < j) {  // + rootpq[j-ma][j-mb] conj(a) u[ma]
      const double rp = c_rpq[(j - ma) * RPQ_STRIDE + col];
      const double ax = rp * a.x, ay = rp * a.y, atx = rp * at.x, aty = rp * at.y;
      const double2 v = s.u[ma], vt = s.t[ma];
      nu.x = fma(ax, v.x, fma(ay, v.y, nu.x));
      nu.y = fma(ax, v.y, fma(-ay, v.x, nu.y));
      nt.x = fma(atx, v.x, fma(aty, v.y, fma(ax, vt.x, fma(ay, vt.y, nt.x))));
      nt.y = fma(atx, v.y, fma(-aty, v.x, fma(ax, vt.y, fma(-ay, vt.x, nt.y))));
    }
    s.u[ma] = nu;
    s.t[ma] = nt;
  }
}

__device__ __forceinline__ double re_cm(double2 x, double2 y) { return fma(x.x, y.x, x.y * y.y); }   // Re(conj(x) y)
__device__ __forceinline__ double im_cm(double2 x, double2 y) { return fma(x.x, y.y, -(x.y * y.x)); }  // Im(conj(x) y)

template <int J, int j>
__device__ __forceinline__ void contract_hvp_lie(const ChainT<J>& s, const double2* __restrict__ yw,
                                                 const double2* __restrict__ yd, int ys, int mb, double (&acc)[12]) {
  const int last = (2 * mb == j) ? mb : j;  // the weighted entries of the row
  const int h0 = half_block(j) + mb * (j + 1);
#pragma unroll
  for (int ma = 0; ma <= j; ma++) {
    if (ma > last) break;
    const double2 w = yw[(h0 + ma) * ys], wd = yd[(h0 + ma) * ys];
    const double2 u = s.u[ma], ut = s.t[ma];
    acc[0] += re_cm(u, w);
    acc[1] += re_cm(ut, w);
    acc[2] += re_cm(u, wd);
    if (j != 2 * ma) {
      const double c = (double)(j - 2 * ma);
      acc[3] = fma(c, im_cm(u, w), acc[3]);
      acc[4] = fma(c, im_cm(ut, w), acc[4]);
      acc[5] = fma(c, im_cm(u, wd), acc[5]);
    }
    // P = s_{ma-1} U[ma-1], Q = s_ma U[ma+1] (and their tangents)
    double2 P = make_double2(0.0, 0.0), Q = P, Pt = P, Qt = P;
    if (ma > 0) {
      const double sg = c_sgen[(j * SGEN_ROWS + mb) * RPQ_STRIDE + ma - 1];
      P = make_double2(sg * s.u[ma - 1].x, sg * s.u[ma - 1].y);
      Pt = make_double2(sg * s.t[ma - 1].x, sg * s.t[ma - 1].y);
    }
    if (ma < j) {
      const double sg = c_sgen[(j * SGEN_ROWS + mb) * RPQ_STRIDE + ma];
      Q = make_double2(sg * s.u[ma + 1].x, sg * s.u[ma + 1].y);
      Qt = make_double2(sg * s.t[ma + 1].x, sg * s.t[ma + 1].y);
    }
    const double2 X = make_double2(P.x - Q.x, P.y - Q.y), Xt = make_double2(Pt.x - Qt.x, Pt.y - Qt.y);
    const double2 Z = make_double2(P.x + Q.x, P.y + Q.y), Zt = make_double2(Pt.x + Qt.x, Pt.y + Qt.y);
    acc[6] += re_cm(X, w);
    acc[7] += re_cm(Xt, w);
    acc[8] += re_cm(X, wd);
    acc[9] += im_cm(Z, w);   // Re(conj(i Z) w) = Im(conj(Z) w)
    acc[10] += im_cm(Zt, w);
    acc[11] += im_cm(Z, wd);
  }
}

template <int J, int j>
__device__ __forceinline__ void save_mirror_t(const ChainT<J>& s, double2* __restrict__ save, int nt, int tid) {
  constexpr int R = (j + 1) / 2;
#pragma unroll
  for (int c = 0; c <= j; c++) {
    const double sg = ((c + R) & 1) ? -1.0 : 1.0;
    const double2 u = s.u[j - c], t = s.t[j - c];
    save[c * nt + tid] = make_double2(sg * u.x, -sg * u.y);
    save[((J + 1) + c) * nt + tid] = make_double2(sg * t.x, -sg * t.y);
  }
}

template <int J, int j>
__device__ __forceinline__ void level_hvp_lie(ChainT<J>& s, double2 a, double2 at, double2 b, double2 bt, int mb,
                                              const double2* yw, const double2* yd, int ys, double (&acc)[12],
                                              double2* save, int nt, int tid) {
  if constexpr (j <= J) {
    advance_t_rt<J, j>(s, a, at, b, bt, mb);
    contract_hvp_lie<J, j>(s, yw, yd, ys, mb, acc);
    if constexpr (j % 2 == 1 && (j + 1) / 2 <= J / 2)
      if (j == 2 * mb + 1) save_mirror_t<J, j>(s, save, nt, tid);  // start row of chain mb+1
  }
}

template <int J>
__device__ __forceinline__ void all_chains_hvp_lie(double2 a, double2 at, double2 b, double2 bt,
                                                   const double2* __restrict__ yw, const double2* __restrict__ yd,
                                                   int ys, double (&acc)[12], double2* save, int nt, int tid) {
  static_assert(J <= 12, "level switch covers twojmax <= 12");
  ChainT<J> s;
#pragma unroll
  for (int c = 0; c <= J; c++) {
    s.u[c] = make_double2(0.0, 0.0);
    s.t[c] = make_double2(0.0, 0.0);
  }
  s.u[0] = make_double2(1.0, 0.0);
#pragma unroll
  for (int q = 0; q < 12; q++) acc[q] = 0.0;
  contract_hvp_lie<J, 0>(s, yw, yd, ys, 0, acc);
#pragma unroll 1
  for (int mb = 0; mb <= J / 2; mb++) {
    if (mb > 0) {
      asm volatile("" ::: "memory");  // this chain's loads stay after the previous chain's saves
#pragma unroll
      for (int c = 0; c <= J; c++) {
        if (c >= 2 * mb) break;
        s.u[c] = save[c * nt + tid];
        s.t[c] = save[((J + 1) + c) * nt + tid];
      }
    }
    switch (mb == 0 ? 1 : 2 * mb) {  // chain mb runs levels 2mb (1 for chain 0) .. J
#define IPG_LEVEL(JJ) \
  case JJ:            \
    level_hvp_lie<J, JJ>(s, a, at, b, bt, mb, yw, yd, ys, acc, save, nt, tid);
      IPG_LEVEL(1) IPG_LEVEL(2) IPG_LEVEL(3) IPG_LEVEL(4) IPG_LEVEL(5) IPG_LEVEL(6)
      IPG_LEVEL(7) IPG_LEVEL(8) IPG_LEVEL(9) IPG_LEVEL(10) IPG_LEVEL(11) IPG_LEVEL(12)
#undef IPG_LEVEL
      default:
        break;
    }
  }
}

}  // namespace snapchain


namespace snapchain {

// ---- every half-plane row of one neighbor handed to an emitter, in chain order ------------
// emit.template row<j>(s, mb) runs after row mb of level j is in registers: row (0, 0) first,
// then chain 0 over levels 1..J, chain mb over levels 2mb..J.  The rows of all lanes of a warp
// come in the same order, so the emitter may synchronise the warp with other warps per row.
template <int J, int j, class Emit>
__device__ __forceinline__ void level_em(Chain<J>& s, const Geom& G, int mb, Emit& emit, double2* save, int nt,
                                         int tid) {
  if constexpr (j <= J) {
    advance_rt<J, j>(s, G, mb);
    emit.template row<j>(s, mb);
    if constexpr (j % 2 == 1 && (j + 1) / 2 <= J / 2)
      if (j == 2 * mb + 1) save_mirror<J, j>(s, save, nt, tid);
  }
}

template <int J, class Emit>
__device__ __forceinline__ void all_chains_rows(const Geom& G, Emit& emit, double2* save, int nt, int tid) {
  static_assert(J <= 12, "level switch covers twojmax <= 12");
  Chain<J> s;
#pragma unroll
  for (int c = 0; c <= J; c++) {
    s.u[c] = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < 3; k++) s.d[k][c] = make_double2(0.0, 0.0);
  }
  s.u[0] = make_double2(1.0, 0.0);
  emit.template row<0>(s, 0);
#pragma unroll 1
  for (int mb = 0; mb <= J / 2; mb++) {
    if (mb > 0) {
      asm volatile("" ::: "memory");
      load_row_rt<J>(s, save, nt, tid, 2 * mb);
    }
    switch (mb == 0 ? 1 : 2 * mb) {
#define IPG_LEVEL(JJ) \
  case JJ:            \
    level_em<J, JJ>(s, G, mb, emit, save, nt, tid);
      IPG_LEVEL(1) IPG_LEVEL(2) IPG_LEVEL(3) IPG_LEVEL(4) IPG_LEVEL(5) IPG_LEVEL(6)
      IPG_LEVEL(7) IPG_LEVEL(8) IPG_LEVEL(9) IPG_LEVEL(10) IPG_LEVEL(11) IPG_LEVEL(12)
#undef IPG_LEVEL
      default:
        break;
    }
  }
}

}  // namespace snapchain

namespace snapchain {

// ---- second order: the tangent of dE_i/dr_ij[k] along a displacement ---------------------
// One (pair, direction k) per thread.  With a dot the derivative along the pair's displacement
// tangent rdot = v_j - v_i, the chain carries U, Udot, dU = dU/dr_k and its tangent dUdot:
//   U_j     = f(a, b, U)
//   Udot_j  = f(adot, bdot, U) + f(a, b, Udot)
//   dU_j    = f(da, db, U) + f(a, b, dU)
//   dUdot_j = f(dadot, dbdot, U) + f(da, db, Udot) + f(adot, bdot, dU) + f(a, b, dUdot)
// with f(A, B, u)[ma] = -rootpq[ma][j-mb] conj(B) u[ma-1] + rootpq[j-ma][j-mb] conj(A) u[ma]
// (the product rule on the recursion of compute_ui.jl:66-101, 224-267), and contracts them
// with the weighted Y of the centre atom and its tangent Ydot:
//   T[0] = sum Re(conj(U) Y),    T[1] = sum Re(conj(dU) Y),    T[2] = sum Re(conj(Udot) Y),
//   T[3] = sum Re(conj(dUdot) Y), T[4] = sum Re(conj(U) Ydot), T[5] = sum Re(conj(dU) Ydot).
template <int J>
struct Chain2 {
  double2 u[J + 1], ut[J + 1], d[J + 1], dt[J + 1];
};
struct Geom2 {
  double2 a, at, b, bt, da, dat, db, dbt;
};

__device__ __forceinline__ void cmac(double2 A, double2 v, double2& acc) {  // acc += conj(A) v
  acc.x = fma(A.x, v.x, fma(A.y, v.y, acc.x));
  acc.y = fma(A.x, v.y, fma(-A.y, v.x, acc.y));
}
__device__ __forceinline__ double2 scl(double r, double2 v) { return make_double2(r * v.x, r * v.y); }

template <int J, int j>
__device__ __forceinline__ void advance2(Chain2<J>& s, const Geom2& G, int mb) {
  const int col = j - mb;
#pragma unroll
  for (int ma = j; ma >= 0; --ma) {
    double2 nu = make_double2(0.0, 0.0), nut = nu, nd = nu, ndt = nu;
    if (ma > 0) {  // - rootpq[ma][j-mb] conj(B) u[ma-1]
      const double rp = -c_rpq[ma * RPQ_STRIDE + col];
      const double2 B = scl(rp, G.b), Bt = scl(rp, G.bt), dB = scl(rp, G.db), dBt = scl(rp, G.dbt);
      const double2 v = s.u[ma - 1], vt = s.ut[ma - 1], dv = s.d[ma - 1], dvt = s.dt[ma - 1];
      cmac(B, v, nu);
      cmac(Bt, v, nut);
      cmac(B, vt, nut);
      cmac(dB, v, nd);
      cmac(B, dv, nd);
      cmac(dBt, v, ndt);
      cmac(dB, vt, ndt);
      cmac(Bt, dv, ndt);
      cmac(B, dvt, ndt);
    }
    if (ma < j) {  // + rootpq[j-ma][j-mb] conj(A) u[ma]
      const double rp = c_rpq[(j - ma) * RPQ_STRIDE + col];
      const double2 A = scl(rp, G.a), At = scl(rp, G.at), dA = scl(rp, G.da), dAt = scl(rp, G.dat);
      const double2 v = s.u[ma], vt = s.ut[ma], dv = s.d[ma], dvt = s.dt[ma];
      cmac(A, v, nu);
      cmac(At, v, nut);
      cmac(A, vt, nut);
      cmac(dA, v, nd);
      cmac(A, dv, nd);
      cmac(dAt, v, ndt);
      cmac(dA, vt, ndt);
      cmac(At, dv, ndt);
      cmac(A, dvt, ndt);
    }
    s.u[ma] = nu;
    s.ut[ma] = nut;
    s.d[ma] = nd;
    s.dt[ma] = ndt;
  }
}

// Yw / Yd point at the centre atom's entry of h = 0 in [h][atom] arrays of stride ys.
template <int J, int j>
__device__ __forceinline__ void contract2(const Chain2<J>& s, const double2* __restrict__ Yw,
                                          const double2* __restrict__ Yd, int64_t ys, int mb, double (&T)[6]) {
  const int last = (2 * mb == j) ? mb : j;  // middle row of an even level stops at ma = j/2
  const int64_t h0 = half_block(j) + mb * (j + 1);
#pragma unroll
  for (int ma = 0; ma <= j; ma++) {
    if (ma > last) break;
    const double2 y = Yw[(h0 + ma) * ys], yd = Yd[(h0 + ma) * ys];
    T[0] = fma(s.u[ma].x, y.x, fma(s.u[ma].y, y.y, T[0]));
    T[1] = fma(s.d[ma].x, y.x, fma(s.d[ma].y, y.y, T[1]));
    T[2] = fma(s.ut[ma].x, y.x, fma(s.ut[ma].y, y.y, T[2]));
    T[3] = fma(s.dt[ma].x, y.x, fma(s.dt[ma].y, y.y, T[3]));
    T[4] = fma(s.u[ma].x, yd.x, fma(s.u[ma].y, yd.y, T[4]));
    T[5] = fma(s.d[ma].x, yd.x, fma(s.d[ma].y, yd.y, T[5]));
  }
}

// Chain mb+1 starts from the mirror of chain mb's row at level 2mb+1 (inversion symmetry,
// compute_ui.jl:105-125), saved as save[(comp (J+1) + c) nt + tid].
template <int J, int j>
__device__ __forceinline__ void save_mirror2(const Chain2<J>& s, double2* __restrict__ save, int nt, int tid) {
  constexpr int R = (j + 1) / 2;
#pragma unroll
  for (int c = 0; c <= j; c++) {
    const double sg = ((c + R) & 1) ? -1.0 : 1.0;
    const double2 src[4] = {s.u[j - c], s.ut[j - c], s.d[j - c], s.dt[j - c]};
#pragma unroll
    for (int q = 0; q < 4; q++) save[(q * (J + 1) + c) * nt + tid] = make_double2(sg * src[q].x, -sg * src[q].y);
  }
}

template <int J>
__device__ __forceinline__ void load_row2(Chain2<J>& s, const double2* __restrict__ save, int nt, int tid, int count) {
#pragma unroll
  for (int c = 0; c <= J; c++) {
    if (c >= count) break;
    s.u[c] = save[(0 * (J + 1) + c) * nt + tid];
    s.ut[c] = save[(1 * (J + 1) + c) * nt + tid];
    s.d[c] = save[(2 * (J + 1) + c) * nt + tid];
    s.dt[c] = save[(3 * (J + 1) + c) * nt + tid];
  }
}

template <int J, int j>
__device__ __forceinline__ void level2(Chain2<J>& s, const Geom2& G, const double2* __restrict__ Yw,
                                       const double2* __restrict__ Yd, int64_t ys, int mb, double (&T)[6],
                                       double2* save, int nt, int tid) {
  if constexpr (j <= J) {
    advance2<J, j>(s, G, mb);
    contract2<J, j>(s, Yw, Yd, ys, mb, T);
    if constexpr (j % 2 == 1 && (j + 1) / 2 <= J / 2)
      if (j == 2 * mb + 1) save_mirror2<J, j>(s, save, nt, tid);
  }
}

// All chains of one (pair, direction): every half-plane entry once (runtime-row level code, as
// all_chains_adjoint).
template <int J>
__device__ __forceinline__ void all_chains_hvp(const Geom2& G, const double2* __restrict__ Yw,
                                               const double2* __restrict__ Yd, int64_t ys, double (&T)[6],
                                               double2* save, int nt, int tid) {
  static_assert(J <= 12, "level switch covers twojmax <= 12");
  Chain2<J> s;
#pragma unroll
  for (int c = 0; c <= J; c++) {
    s.u[c] = make_double2(0.0, 0.0);
    s.ut[c] = s.u[c];
    s.d[c] = s.u[c];
    s.dt[c] = s.u[c];
  }
  s.u[0] = make_double2(1.0, 0.0);  // level 0: U = 1, every derivative and tangent 0
#pragma unroll
  for (int q = 0; q < 6; q++) T[q] = 0.0;
  contract2<J, 0>(s, Yw, Yd, ys, 0, T);
#pragma unroll 1
  for (int mb = 0; mb <= J / 2; mb++) {
    if (mb > 0) {
      asm volatile("" ::: "memory");  // this chain's loads stay after the previous chain's saves
      load_row2<J>(s, save, nt, tid, 2 * mb);  // row mb of level 2mb-1
    }
    switch (mb == 0 ? 1 : 2 * mb) {  // chain mb runs levels 2mb (1 for chain 0) .. J
#define IPG_LEVEL(JJ) \
  case JJ:            \
    level2<J, JJ>(s, G, Yw, Yd, ys, mb, T, save, nt, tid);
      IPG_LEVEL(1) IPG_LEVEL(2) IPG_LEVEL(3) IPG_LEVEL(4) IPG_LEVEL(5) IPG_LEVEL(6)
      IPG_LEVEL(7) IPG_LEVEL(8) IPG_LEVEL(9) IPG_LEVEL(10) IPG_LEVEL(11) IPG_LEVEL(12)
#undef IPG_LEVEL
      default:
        break;
    }
  }
}

}  // namespace snapchain
