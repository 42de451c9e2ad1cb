// ipg_pair.cu — fused multi-term empirical pair potentials.
//
// Replaces, for every term of a LinearCombinationPotential at once, the per-term
// neighbor build + pair loop of src/types/empirical_potential.jl:20-67 with one walk of
// the cell list at the largest cutoff.  One thread owns one atom (cell-sorted order, so a
// warp reads the same neighbor cells), visits every candidate once, and applies each
// term's own cutoff (PeriodicEuclidean distance <= rcut_t, as the term's own neighbor
// list would) and species filter (both species in the term's set,
// empirical_potential.jl:26-43).  Each atom sums its full neighbor set, so forces need no
// atomics; the half-list energy and virial are recovered as 1/2 of the directed sums.
// For j < i the displacement is the negated reference displacement of the stored half
// pair (i.e. -get_displacement(x_j, x_i)), so every force term equals the reference's
// term bit for bit; only the order of summation differs.
#include "ipg_internal.cuh"

namespace {

struct PairTermDev {
  int kind;
  int pad;
  double coeff, rcut;
  unsigned long long mask;
  double p[8];  // kind-specific precomputed constants (see prepare_terms)
};

struct PairTerms {
  int nterms;
  double rcut_max;
  double rmax2_hi;  // rcut_max^2 (1 + 1e-12): candidates beyond it are out for sure
  PairTermDev t[IPG_MAX_PAIR_TERMS];
};

static_assert(sizeof(PairTerms) <= 4096, "the terms travel as a kernel parameter");

// ZBL screening coefficients, src/empirical/zbl.jl:27-28.
__constant__ double c_zbl_c[4] = {0.18175, 0.50986, 0.28022, 0.02817};
__constant__ double c_zbl_a[4] = {3.19980, 0.94229, 0.40290, 0.20162};

// V(R) and g(R) (force = g r) of one term.
__device__ __forceinline__ void term_eval(const PairTermDev& t, double R, double& V, double& g) {
  switch (t.kind) {
    case IPG_PAIR_LJ: {  // lj.jl:35-36; p = eps, sigma, 4eps, 24eps
      double s = t.p[1] / R;
      double s2 = s * s;
      double s6 = s2 * s2 * s2;
      double s12 = s6 * s6;
      V = t.p[2] * (s12 - s6);
      g = t.p[3] * (2.0 * s12 - s6) / (R * R);
      break;
    }
    case IPG_PAIR_BM: {  // bm.jl:38-39; p = A, rho, sigma, C, D
      double ex = t.p[0] * exp((t.p[2] - R) / t.p[1]);
      double c = t.p[3] / R, d = t.p[4] / R;
      double c2 = c * c, d2 = d * d;
      double c6 = c2 * c2 * c2, d8 = (d2 * d2) * (d2 * d2);
      V = ex + c6 - d8;
      g = ex / (t.p[1] * R) + (c6 - d8) / (R * R);
      break;
    }
    case IPG_PAIR_COUL: {  // coulomb.jl:36-37; p = q1, q2, k_e q1 q2
      V = t.p[2] / R;
      g = t.p[2] / (R * R * R);
      break;
    }
    case IPG_PAIR_MORSE: {  // morse.jl:36-39; p = D, alpha, sigma
      double e = exp(-t.p[1] * (R - t.p[2]));
      double om = 1.0 - e;
      V = t.p[0] * om * om;
      g = 2.0 * t.p[0] * t.p[1] * om * e / R;
      break;
    }
    case IPG_PAIR_ZBL: {  // zbl.jl:29-36; p = Z1, Z2, e, coeff = Z1 Z2 e^2, dden, ln(e)
      double d = R / t.p[4];
      double phi = 0.0, dphi = 0.0;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        double ek = exp(-c_zbl_a[k] * d * t.p[5]);  // e^(-a_k d) with base e = p[2]
        phi += c_zbl_c[k] * ek;
        dphi += c_zbl_a[k] * c_zbl_c[k] * ek;
      }
      dphi = -dphi;
      V = t.p[3] * phi / R;
      g = t.p[3] * (phi + d * dphi) / (R * R * R);
      break;
    }
    case IPG_PAIR_MOCK_R2: {  // test/mocks.jl:29-34; p = seed
      V = R * R * t.p[0];
      g = R * R * t.p[0];
      break;
    }
    default:
      V = 0.0;
      g = 0.0;
  }
}

constexpr int PAIR_T = 128;
constexpr int PAIR_WARPS = PAIR_T / 32;

// One warp per atom (cell-sorted order).  Lanes test consecutive candidates of each
// stencil range; the pairs within the largest cutoff are compacted into a per-warp
// shared buffer (ballot prefix, candidate order), and every 32 of them are evaluated by
// the whole warp, so the term arithmetic (exp, pow) runs on full warps.
struct Hit {
  double r0, r1, r2, dist;
  int sj, pad;
};

__device__ __forceinline__ void eval_hits(const PairTerms& TT, const Hit* __restrict__ hb, int nh, int lane, int si,
                                          double* acc, double& f0, double& f1, double& f2) {
  if (lane >= nh) return;
  const Hit h = hb[lane];
  const double R = sqrt(h.r0 * h.r0 + h.r1 * h.r1 + h.r2 * h.r2);
  double V = 0.0, gsum = 0.0;
  for (int t = 0; t < TT.nterms; t++) {
    const PairTermDev& T = TT.t[t];
    if (h.dist > T.rcut) continue;
    if (!((T.mask >> si) & 1ull) || !((T.mask >> h.sj) & 1ull)) continue;
    double v, gg;
    term_eval(T, R, v, gg);
    V += T.coeff * v;
    gsum += T.coeff * gg;
  }
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

__global__ void __launch_bounds__(PAIR_T) k_pair_eval(const __grid_constant__ PairTerms TT, int64_t n,
                                                      const ConfGrid* __restrict__ grid,
                                                      const int64_t* __restrict__ cell_start,
                                                      const int32_t* __restrict__ cell_atoms,
                                                      const double4* __restrict__ spos, double* __restrict__ F,
                                                      double* __restrict__ partial, int* status) {
  __shared__ Hit hits[PAIR_WARPS][64];
  __shared__ double red[PAIR_WARPS][7];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t s = (int64_t)blockIdx.x * PAIR_WARPS + w;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};  // E, W[6]
  if (s < n) {  // warp-uniform
    const int32_t i = cell_atoms[s];
    const double4 xi = spos[s];
    const int si = (int)xi.w;
    const ConfGrid g = grid[0];
    int c[3];
    cell_coords(g, xi.x, xi.y, xi.z, c);
    StencilRanges Rg;
    stencil_ranges(g, c, cell_start, Rg);
    double f0 = 0.0, f1 = 0.0, f2 = 0.0;
    const double rmax = TT.rcut_max;
    Hit* hb = hits[w];
    int nh = 0;
    const unsigned lt = (1u << lane) - 1u;
    for (int r = 0; r < Rg.n; r++)
      for (int64_t q0 = Rg.beg[r]; q0 < Rg.end[r]; q0 += 32) {
        const int64_t q = q0 + lane;
        bool ok = false;
        Hit h;
        if (q < Rg.end[r]) {
          const int32_t j = cell_atoms[q];
          const double4 xj = spos[q];
          if (j != i) {
            const double p0 = pe_axis_dev(g.L[0], xi.x, xj.x);
            const double p1 = pe_axis_dev(g.L[1], xi.y, xj.y);
            const double p2 = pe_axis_dev(g.L[2], xi.z, xj.z);
            const double d2 = sumsq3_dev(p0, p1, p2);
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
        if (nh >= 32) {
          eval_hits(TT, hb, 32, lane, si, acc, f0, f1, f2);
          __syncwarp();
          if (lane < nh - 32) hb[lane] = hb[32 + lane];
          nh -= 32;
          __syncwarp();
        }
      }
    eval_hits(TT, hb, nh, lane, si, acc, f0, f1, f2);
    f0 = warp_sum(f0);
    f1 = warp_sum(f1);
    f2 = warp_sum(f2);
    if (F && lane == 0) {
      F[3 * (int64_t)i] = f0;
      F[3 * (int64_t)i + 1] = f1;
      F[3 * (int64_t)i + 2] = f2;
    }
  }
#pragma unroll
  for (int k = 0; k < 7; k++) {
    double v = warp_sum(acc[k]);
    if (lane == 0) red[w][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < 7) {
    double v = 0.0;
    for (int q = 0; q < PAIR_WARPS; q++) v += red[q][threadIdx.x];
    partial[(int64_t)blockIdx.x * 7 + threadIdx.x] = v;
  }
}

// Deterministic final reduction of per-block partials: one block, fixed order.
__global__ void k_reduce_partials(int64_t nblocks, int width, const double* __restrict__ partial,
                                  double* __restrict__ out) {
  __shared__ double sm[256];
  for (int k = 0; k < width; k++) {
    double v = 0.0;
    for (int64_t b = threadIdx.x; b < nblocks; b += blockDim.x) v += partial[b * width + k];
    sm[threadIdx.x] = v;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if ((int)threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[k] = sm[0];
    __syncthreads();
  }
}

int prepare_terms(ipg_ctx* ctx, const ipg_pair_term* terms, int nterms, PairTerms& pt) {
  memset(&pt, 0, sizeof(pt));
  if (nterms < 0 || nterms > IPG_MAX_PAIR_TERMS)
    return ipg_fail(ctx, IPG_ERR_ARG, "nterms must be in 0..%d", IPG_MAX_PAIR_TERMS);
  pt.nterms = nterms;
  pt.rcut_max = 0.0;
  pt.rmax2_hi = 0.0;
  for (int k = 0; k < nterms; k++) {
    const ipg_pair_term& s = terms[k];
    PairTermDev& d = pt.t[k];
    d.kind = s.kind;
    d.coeff = s.coeff;
    d.rcut = s.rcut;
    d.mask = s.species_mask;
    if (!(s.rcut >= 0.0)) return ipg_fail(ctx, IPG_ERR_ARG, "term %d: rcut must be >= 0", k);
    if (std::isinf(s.rcut)) return ipg_fail(ctx, IPG_ERR_ARG, "term %d: rcut must be finite", k);
    pt.rcut_max = std::max(pt.rcut_max, s.rcut);
    for (int q = 0; q < 8; q++) d.p[q] = s.params[q];
    switch (s.kind) {
      case IPG_PAIR_LJ:
        d.p[2] = 4.0 * s.params[0];
        d.p[3] = 24.0 * s.params[0];
        break;
      case IPG_PAIR_BM:
      case IPG_PAIR_MORSE:
      case IPG_PAIR_MOCK_R2:
        break;
      case IPG_PAIR_COUL:
        d.p[2] = 1.0 * s.params[0] * s.params[1];  // k_e = 1 (src/constants.jl:7)
        break;
      case IPG_PAIR_ZBL: {
        double Z1 = s.params[0], Z2 = s.params[1], e = s.params[2];
        d.p[3] = 1.0 * Z1 * Z2 * e * e;                                     // _zbl_coeff
        d.p[4] = 0.8854 * 0.529 / (std::pow(Z1, 0.23) + std::pow(Z2, 0.23));  // _zbl_d divisor
        d.p[5] = std::log(e);
        if (!(e > 0.0)) return ipg_fail(ctx, IPG_ERR_ARG, "term %d: ZBL e must be > 0", k);
        break;
      }
      default:
        return ipg_fail(ctx, IPG_ERR_ARG, "term %d: unknown kind %d", k, s.kind);
    }
  }
  pt.rmax2_hi = pt.rcut_max * pt.rcut_max * (1.0 + 1e-12);
  return IPG_OK;
}

int pair_eval_device(ipg_ctx* ctx, int64_t n, const double* d_pos, const int32_t* d_species, const double L[3],
                     const ipg_pair_term* terms, int32_t nterms, double* d_E, double* d_F, double* d_W6,
                     uint32_t flags) {
  PairTerms pt;
  IPG_RET(prepare_terms(ctx, terms, nterms, pt));
  IPG_RET(ipg_status_reset(ctx));
  int64_t aoff[2] = {0, n};
  CellList cl;
  IPG_RET(ipg_build_cells(ctx, "pair_", n, d_pos, d_species, 64, 1, aoff, L, pt.rcut_max, cl));
  int64_t nb = std::max<int64_t>(1, (n + PAIR_WARPS - 1) / PAIR_WARPS);
  double *partial, *red;
  IPG_RET(scratch(ctx, "pair_partial", (size_t)nb * 7, &partial));
  IPG_RET(scratch(ctx, "pair_red", 8, &red));
  IPG_TIMED_LAUNCH(ctx, "pair_eval", k_pair_eval, (unsigned)nb, PAIR_T, 0, pt, n, cl.d_grid, cl.d_cell_start, cl.d_cell_atoms, cl.d_spos,
             (flags & IPG_WANT_F) ? d_F : nullptr, partial, ctx->d_status);
  IPG_LAUNCH(ctx, k_reduce_partials, 1, 256, 0, nb, 7, partial, red);
  if ((flags & IPG_WANT_E) && d_E)
    CUDA_RET(ctx, cudaMemcpyAsync(d_E, red, sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  if ((flags & IPG_WANT_W) && d_W6)
    CUDA_RET(ctx, cudaMemcpyAsync(d_W6, red + 1, 6 * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  return IPG_OK;
}

int check_pair_args(ipg_ctx* ctx, int64_t n, const void* pos, const void* species, const double* L,
                    const ipg_pair_term* terms, int32_t nterms, const void* E, const void* F, const void* W6,
                    uint32_t flags) {
  if (!ctx) return IPG_ERR_ARG;
  if (n < 0 || n >= INT32_MAX) return ipg_fail(ctx, IPG_ERR_ARG, "n out of range");
  if ((n > 0 && (!pos || !species)) || !L || (nterms > 0 && !terms))
    return ipg_fail(ctx, IPG_ERR_ARG, "null input pointer");
  if ((flags & IPG_WANT_E) && !E) return ipg_fail(ctx, IPG_ERR_ARG, "E requested but NULL");
  if ((flags & IPG_WANT_F) && !F && n > 0) return ipg_fail(ctx, IPG_ERR_ARG, "F requested but NULL");
  if ((flags & IPG_WANT_W) && !W6) return ipg_fail(ctx, IPG_ERR_ARG, "W6 requested but NULL");
  return IPG_OK;
}

}  // namespace

extern "C" {

int ipg_pair_eval(ipg_ctx* ctx, int64_t n, const double* pos, const int32_t* species, const double L[3],
                  const ipg_pair_term* terms, int32_t nterms, double* E, double* F, double* W6, uint32_t flags) {
  IPG_RET(check_pair_args(ctx, n, pos, species, L, terms, nterms, E, F, W6, flags));
  CUDA_RET(ctx, cudaSetDevice(ctx->device));
  if (!host_all_finite(pos, 3 * n)) return ipg_fail(ctx, IPG_ERR_NONFINITE, "non-finite position");
  if (!host_species_ok(species, n, 64)) return ipg_fail(ctx, IPG_ERR_SPECIES, "species id out of range 0..63");
  double *d_pos, *d_out;
  int32_t* d_sp;
  IPG_RET(scratch(ctx, "pair_in_pos", 3 * (size_t)n + 3, &d_pos));
  IPG_RET(scratch(ctx, "pair_in_sp", (size_t)n + 1, &d_sp));
  IPG_RET(scratch(ctx, "pair_out", 3 * (size_t)n + 8, &d_out));
  if (n) {
    CUDA_RET(ctx, cudaMemcpyAsync(d_pos, pos, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_RET(ctx, cudaMemcpyAsync(d_sp, species, sizeof(int32_t) * n, cudaMemcpyHostToDevice, ctx->stream));
  }
  // d_out layout: [E, W6 (6), pad, F (3n)]
  IPG_RET(pair_eval_device(ctx, n, d_pos, d_sp, L, terms, nterms, d_out, d_out + 8, d_out + 1,
                           flags | IPG_WANT_E | IPG_WANT_W));
  std::vector<double> head(8);
  CUDA_RET(ctx, cudaMemcpyAsync(head.data(), d_out, sizeof(double) * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if ((flags & IPG_WANT_F) && n)
    CUDA_RET(ctx, cudaMemcpyAsync(F, d_out + 8, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, ctx->stream));
  IPG_RET(ipg_status_check(ctx, "ipg_pair_eval"));
  if (flags & IPG_WANT_E) *E = head[0];
  if (flags & IPG_WANT_W) memcpy(W6, head.data() + 1, 6 * sizeof(double));
  return IPG_OK;
}

int ipg_pair_eval_dev(ipg_ctx* ctx, int64_t n, const double* d_pos, const int32_t* d_species, const double L[3],
                      const ipg_pair_term* terms, int32_t nterms, double* d_E, double* d_F, double* d_W6,
                      uint32_t flags) {
  IPG_RET(check_pair_args(ctx, n, d_pos, d_species, L, terms, nterms, d_E, d_F, d_W6, flags));
  CUDA_RET(ctx, cudaSetDevice(ctx->device));
  IPG_RET(pair_eval_device(ctx, n, d_pos, d_species, L, terms, nterms, d_E, d_F, d_W6, flags));
  IPG_RET(ipg_status_check(ctx, "ipg_pair_eval_dev"));
  return IPG_OK;
}

}  // extern "C"
