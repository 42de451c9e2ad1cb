// ipg_pair.cuh — the empirical pair terms and the full-stencil pair walk, shared by the
// context path (ipg_pair.cu) and the no-allocation path (ipg_noalloc.cu).
//
// The five pair formulas follow the reference literally (src/empirical/{lj,bm,coulomb,
// morse,zbl}.jl and test/mocks.jl), quirks included: Born–Mayer's (C/R)^6 and (D/R)^8
// force terms without their 6 and 8, Morse's force along +grad V, ZBL's screening with base
// e (the charge parameter) and a force that is not -grad V.
#pragma once

#include <algorithm>

#include "ipg_internal.cuh"

struct PairTermDev {
  int kind;
  int pad;
  double coeff, rcut;
  unsigned long long mask;
  double p[8];  // kind-specific precomputed constants (see pair_prepare_terms)
};

struct PairTerms {
  int nterms;
  double rcut_max;
  double rmax2_hi;  // rcut_max^2 (1 + 1e-12): candidates beyond it are out for sure
  PairTermDev t[IPG_MAX_PAIR_TERMS];
};

static_assert(sizeof(PairTerms) <= 4096, "the terms travel as a kernel parameter");

// Host: the kernel-side terms of an ipg_pair_term list.  Returns IPG_OK or IPG_ERR_ARG with a
// message in err.
inline int pair_prepare_terms(const ipg_pair_term* terms, int nterms, PairTerms& pt, char* err, size_t errlen) {
  memset(&pt, 0, sizeof(pt));
  if (nterms < 0 || nterms > IPG_MAX_PAIR_TERMS) {
    snprintf(err, errlen, "nterms must be in 0..%d", IPG_MAX_PAIR_TERMS);
    return IPG_ERR_ARG;
  }
  pt.nterms = nterms;
  for (int k = 0; k < nterms; k++) {
    const ipg_pair_term& s = terms[k];
    PairTermDev& d = pt.t[k];
    d.kind = s.kind;
    d.coeff = s.coeff;
    d.rcut = s.rcut;
    d.mask = s.species_mask;
    if (!(s.rcut >= 0.0) || std::isinf(s.rcut)) {
      snprintf(err, errlen, "term %d: rcut must be finite and >= 0", k);
      return IPG_ERR_ARG;
    }
    pt.rcut_max = std::max(pt.rcut_max, s.rcut);
    for (int q = 0; q < 8; q++) d.p[q] = s.params[q];
    switch (s.kind) {
      case IPG_PAIR_LJ:  // p = eps, sigma, 4 eps, 24 eps
        d.p[2] = 4.0 * s.params[0];
        d.p[3] = 24.0 * s.params[0];
        break;
      case IPG_PAIR_BM:  // p = A, rho, sigma, C, D, 1/rho
        d.p[5] = 1.0 / s.params[1];
        break;
      case IPG_PAIR_MORSE:
      case IPG_PAIR_MOCK_R2:
        break;
      case IPG_PAIR_COUL:  // p = q1, q2, k_e q1 q2 with k_e = 1 (src/constants.jl:7)
        d.p[2] = 1.0 * s.params[0] * s.params[1];
        break;
      case IPG_PAIR_ZBL: {  // p = Z1, Z2, e, Z1 Z2 e^2, the screening length, ln(e), 1/length
        const double Z1 = s.params[0], Z2 = s.params[1], e = s.params[2];
        if (!(e > 0.0)) {
          snprintf(err, errlen, "term %d: ZBL e must be > 0", k);
          return IPG_ERR_ARG;
        }
        d.p[3] = 1.0 * Z1 * Z2 * e * e;
        d.p[4] = 0.8854 * 0.529 / (std::pow(Z1, 0.23) + std::pow(Z2, 0.23));
        d.p[5] = std::log(e);
        d.p[6] = 1.0 / d.p[4];
        break;
      }
      default:
        snprintf(err, errlen, "term %d: unknown kind %d", k, s.kind);
        return IPG_ERR_ARG;
    }
  }
  pt.rmax2_hi = pt.rcut_max * pt.rcut_max * (1.0 + 1e-12);
  return IPG_OK;
}

// V(R) and g(R) (force = g r) of one term; ir = 1/R and ir2 = 1/R^2 are formed once per pair,
// so every division by R of the reference formulas is a product with ir (the results differ
// from the literal divisions by rounding only).
__device__ __forceinline__ void pair_term_eval(const PairTermDev& t, double R, double ir, double ir2, double& V,
                                               double& g) {
  switch (t.kind) {
    case IPG_PAIR_LJ: {  // lj.jl:35-36; p = eps, sigma, 4 eps, 24 eps
      const double s = t.p[1] * ir;
      const double s2 = s * s;
      const double s6 = s2 * s2 * s2;
      const double s12 = s6 * s6;
      V = t.p[2] * (s12 - s6);
      g = t.p[3] * (2.0 * s12 - s6) * ir2;
      break;
    }
    case IPG_PAIR_BM: {  // bm.jl:38-39; p = A, rho, sigma, C, D, 1/rho
      const double ex = t.p[0] * exp((t.p[2] - R) * t.p[5]);
      const double c = t.p[3] * ir, d = t.p[4] * ir;
      const double c2 = c * c, d2 = d * d;
      const double c6 = c2 * c2 * c2, d8 = (d2 * d2) * (d2 * d2);
      V = ex + c6 - d8;
      g = ex * t.p[5] * ir + (c6 - d8) * ir2;
      break;
    }
    case IPG_PAIR_COUL:  // coulomb.jl:36-37; p = q1, q2, k_e q1 q2
      V = t.p[2] * ir;
      g = t.p[2] * ir * ir2;
      break;
    case IPG_PAIR_MORSE: {  // morse.jl:36-39; p = D, alpha, sigma
      const double e = exp(-t.p[1] * (R - t.p[2]));
      const double om = 1.0 - e;
      V = t.p[0] * om * om;
      g = 2.0 * t.p[0] * t.p[1] * om * e * ir;
      break;
    }
    case IPG_PAIR_ZBL: {  // zbl.jl:27-36: e^(-a_k d) with base e = p[2]
      const double zc[4] = {0.18175, 0.50986, 0.28022, 0.02817};
      const double za[4] = {3.19980, 0.94229, 0.40290, 0.20162};
      const double d = R * t.p[6];
      double phi = 0.0, dphi = 0.0;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const double ek = exp(-za[k] * d * t.p[5]);
        phi += zc[k] * ek;
        dphi += za[k] * zc[k] * ek;
      }
      dphi = -dphi;
      V = t.p[3] * phi * ir;
      g = t.p[3] * (phi + d * dphi) * ir * ir2;
      break;
    }
    case IPG_PAIR_MOCK_R2:  // test/mocks.jl:29-34; p = seed
      V = R * R * t.p[0];
      g = R * R * t.p[0];
      break;
    default:
      V = 0.0;
      g = 0.0;
  }
}

// Sum of c_t V_t and c_t g_t over the terms that apply to a pair (distance `dist` for the
// cutoffs, R = |r| for the formulas, species si and sj for the filters:
// src/types/empirical_potential.jl:26-43, both species in the term's set).
__device__ __forceinline__ void pair_terms_sum(const PairTerms& TT, double R, double dist, int si, int sj, double& V,
                                               double& g) {
  V = 0.0;
  g = 0.0;
  const double ir = 1.0 / R, ir2 = ir * ir;
  for (int t = 0; t < TT.nterms; t++) {
    const PairTermDev& T = TT.t[t];
    if (dist > T.rcut) continue;
    if (!((T.mask >> si) & 1ull) || !((T.mask >> sj) & 1ull)) continue;
    double v, gg;
    pair_term_eval(T, R, ir, ir2, v, gg);
    V += T.coeff * v;
    g += T.coeff * gg;
  }
}

// ---------------------------------------------------------------------------------
// Full-stencil walk: one warp per atom over its 27-cell stencil.  Lanes test consecutive
// candidates of each stencil range; the pairs within the largest cutoff are compacted into a
// per-warp shared buffer (ballot prefix, candidate order) and every 32 of them are evaluated
// by the whole warp.  Each atom sums its full neighbor set (so its force needs no other warp);
// the half-list energy and virial are 1/2 of the directed sums.  For j < i the displacement
// is the negated reference displacement of the stored half pair, -get_displacement(x_j, x_i),
// so every force term equals the reference's term; only the order of summation differs.
struct PairHit {
  double r0, r1, r2, dist;
  int sj, pad;
};

__device__ __forceinline__ void pair_eval_hits(const PairTerms& TT, const PairHit* __restrict__ hb, int nh, int lane,
                                               int si, double* acc, double& f0, double& f1, double& f2) {
  if (lane >= nh) return;
  const PairHit h = hb[lane];
  const double R = sqrt(h.r0 * h.r0 + h.r1 * h.r1 + h.r2 * h.r2);
  double V, gsum;
  pair_terms_sum(TT, R, h.dist, si, h.sj, V, gsum);
  const double fx = gsum * h.r0, fy = gsum * h.r1, fz = gsum * h.r2;
  f0 += fx;
  f1 += fy;
  f2 += fz;
  acc[0] += 0.5 * V;
  // empirical_potential.jl:63-64: r * f' -> [xx, yy, zz, zy, zx, yx]
  acc[1] += 0.5 * h.r0 * fx;
  acc[2] += 0.5 * h.r1 * fy;
  acc[3] += 0.5 * h.r2 * fz;
  acc[4] += 0.5 * h.r2 * fy;
  acc[5] += 0.5 * h.r2 * fx;
  acc[6] += 0.5 * h.r1 * fx;
}

// The walk of the atom in slot s; hb is this warp's buffer of 64 hits.  Adds the atom's half
// of E and W to acc (lane-wise) and writes its force to F (original atom order) if F != null.
__device__ __forceinline__ void pair_walk_atom(const PairTerms& TT, const ConfGrid& g,
                                               const int64_t* __restrict__ cell_start,
                                               const int32_t* __restrict__ cell_atoms,
                                               const double4* __restrict__ spos, int64_t s, PairHit* hb, int lane,
                                               double* acc, double* __restrict__ F) {
  const int32_t i = cell_atoms[s];
  const double4 xi = spos[s];
  const int si = (int)xi.w;
  int c[3];
  cell_coords(g, xi.x, xi.y, xi.z, c);
  StencilRanges Rg;
  stencil_ranges(g, c, cell_start, Rg);
  double f0 = 0.0, f1 = 0.0, f2 = 0.0;
  const double rmax = TT.rcut_max;
  int nh = 0;
  const unsigned lt = (1u << lane) - 1u;
  for (int r = 0; r <= Rg.n; r++)  // r == Rg.n: evaluate what is left
    for (int64_t q0 = r < Rg.n ? Rg.beg[r] : 0; q0 < (r < Rg.n ? Rg.end[r] : 1); q0 += 32) {
      const int64_t q = q0 + lane;
      bool ok = false;
      PairHit h;
      if (r < Rg.n && q < Rg.end[r]) {
        const int32_t j = cell_atoms[q];
        const double4 xj = spos[q];
        if (j != i) {
          const double d2 = sumsq3_dev(pe_axis_dev(g.L[0], xi.x, xj.x), pe_axis_dev(g.L[1], xi.y, xj.y),
                                       pe_axis_dev(g.L[2], xi.z, xj.z));
          if (d2 <= TT.rmax2_hi) {
            const double dist = sqrt(d2);
            if (dist <= rmax) {
              ok = true;
              h.dist = dist;
              h.sj = (int)xj.w;
              if (j > i) {
                h.r0 = disp_axis_dev(g.L[0], xi.x, xj.x);
                h.r1 = disp_axis_dev(g.L[1], xi.y, xj.y);
                h.r2 = disp_axis_dev(g.L[2], xi.z, xj.z);
              } else {  // -get_displacement(x_j, x_i): the reference's stored half pair
                h.r0 = -disp_axis_dev(g.L[0], xj.x, xi.x);
                h.r1 = -disp_axis_dev(g.L[1], xj.y, xi.y);
                h.r2 = -disp_axis_dev(g.L[2], xj.z, xi.z);
              }
            }
          }
        }
      }
      const unsigned bal = __ballot_sync(0xffffffffu, ok);
      if (ok) hb[nh + __popc(bal & lt)] = h;
      nh += __popc(bal);
      __syncwarp();
      // one call site of the term code: full batches, then the rest after the last range
      while (nh >= 32 || (r == Rg.n && nh > 0)) {
        const int m = nh < 32 ? nh : 32;
        pair_eval_hits(TT, hb, m, lane, si, acc, f0, f1, f2);
        __syncwarp();
        if (lane < nh - m) hb[lane] = hb[m + lane];
        nh -= m;
        __syncwarp();
      }
    }
  f0 = warp_sum(f0);
  f1 = warp_sum(f1);
  f2 = warp_sum(f2);
  if (F && lane == 0) {
    F[3 * (int64_t)i] = f0;
    F[3 * (int64_t)i + 1] = f1;
    F[3 * (int64_t)i + 2] = f2;
  }
}
