// ipg_oracle.cpp — CPU restatement of InteratomicPotentials.jl's force-field hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library: only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.  The
// product path (libipg.so) never links or calls it.
//
// Every function restates the reference Julia loop it names (file:line within
// cesmix-mit/InteratomicPotentials.jl v0.3.2), with 0-based indices.  Arithmetic is
// FP64 and the file is compiled with -ffp-contract=off so that no multiply-add is
// fused behind the reader's back.
//
// Neighbor search: the reference uses a NearestNeighbors.jl BallTree with a
// Distances.jl PeriodicEuclidean metric (src/nnlist.jl:30-40,
// src/BasisSystems/SNAP/utilities/utl.jl:65-81).  The tree only proposes candidates;
// membership is decided by the metric, so this restatement proposes candidates from a
// cell list (complete for any cell edge >= search radius) and applies the same
// per-candidate test.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// Julia `mod(x, y)` for Float64 (result takes the sign of y).
inline double jl_mod(double x, double y) {
  if (std::isinf(y)) return (x >= 0.0) ? x : y;  // mod(x, Inf) for finite x>=0 is x
  double r = std::fmod(x, y);
  if (r == 0.0) return std::copysign(0.0, y);
  if ((r > 0.0) != (y > 0.0)) r += y;
  return r;
}

// src/nnlist.jl:18-21 get_displacement (== utl.jl:27-36 get_distance): x - y under
// minimum image on periodic axes, plain difference where L is Inf.
inline double disp_axis(double L, double x, double y) {
  if (std::isinf(L)) return x - y;
  double d = jl_mod(x - y, L);
  return (2.0 * d < L) ? d : d - L;
}

// Distances.jl PeriodicEuclidean per-axis term (abs, mod, min with the far image).
inline double pe_axis(double L, double a, double b) {
  double s1 = std::fabs(a - b);
  if (std::isinf(L)) return s1;
  double s2 = jl_mod(s1, L);
  return std::min(s2, L - s2);
}

inline double pe_dist(const double* L, const double* a, const double* b) {
  double s0 = pe_axis(L[0], a[0], b[0]);
  double s1 = pe_axis(L[1], a[1], b[1]);
  double s2 = pe_axis(L[2], a[2], b[2]);
  double s = s0 * s0;
  s = s + s1 * s1;
  s = s + s2 * s2;
  return std::sqrt(s);
}

// ---------------------------------------------------------------------------------
// Candidate generator: a cell list over wrapped coordinates.  cand(n) lists every atom
// m (m != n) that can lie within `radius` of atom n, each once, in ascending order.
struct CellGrid {
  int nc[3];
  double lo[3], cs[3];
  bool per[3];
  std::vector<int64_t> cell_start;
  std::vector<int64_t> order;
  std::vector<int> cell_of;
};

bool build_grid(CellGrid& g, int64_t n, const double* pos, const double* L, double radius) {
  double rc = radius * (1.0 + 1e-9);
  double ext[3];
  int64_t total = 1;
  for (int a = 0; a < 3; a++) {
    g.per[a] = !std::isinf(L[a]);
    double lo = 0.0, hi = 0.0;
    if (g.per[a]) {
      hi = L[a];
    } else if (n > 0) {
      lo = std::numeric_limits<double>::infinity();
      hi = -lo;
      for (int64_t i = 0; i < n; i++) {
        lo = std::min(lo, pos[3 * i + a]);
        hi = std::max(hi, pos[3 * i + a]);
      }
    }
    g.lo[a] = lo;
    ext[a] = hi - lo;
    int nc = 1;
    if (rc > 0.0 && std::isfinite(rc) && ext[a] > 0.0) nc = (int)std::max(1.0, std::min(std::floor(ext[a] / rc), 1024.0));
    g.nc[a] = nc;
    total *= nc;
  }
  while (total > std::max<int64_t>(64, 8 * n)) {  // keep the grid proportional to n
    int a = (g.nc[0] >= g.nc[1] && g.nc[0] >= g.nc[2]) ? 0 : (g.nc[1] >= g.nc[2] ? 1 : 2);
    total /= g.nc[a];
    g.nc[a] = std::max(1, g.nc[a] / 2);
    total *= g.nc[a];
  }
  for (int a = 0; a < 3; a++) g.cs[a] = (ext[a] > 0.0) ? ext[a] / g.nc[a] : 1.0;
  int64_t ncell = total;
  g.cell_of.assign(n, 0);
  std::vector<int64_t> count(ncell + 1, 0);
  for (int64_t i = 0; i < n; i++) {
    int c[3];
    for (int a = 0; a < 3; a++) {
      double x = pos[3 * i + a];
      double w = g.per[a] ? x - L[a] * std::floor(x / L[a]) : x - g.lo[a];
      int k = (int)std::floor(w / g.cs[a]);
      c[a] = std::min(std::max(k, 0), g.nc[a] - 1);
    }
    int cell = (c[2] * g.nc[1] + c[1]) * g.nc[0] + c[0];
    g.cell_of[i] = cell;
    count[cell + 1]++;
  }
  for (int64_t c = 0; c < ncell; c++) count[c + 1] += count[c];
  g.cell_start = count;
  g.order.assign(n, 0);
  std::vector<int64_t> fill(count.begin(), count.end() - 1);
  for (int64_t i = 0; i < n; i++) g.order[fill[g.cell_of[i]]++] = i;
  return true;
}

void candidates(const CellGrid& g, int64_t n_atom, std::vector<int64_t>& out) {
  out.clear();
  int cell = g.cell_of[n_atom];
  int c[3] = {cell % g.nc[0], (cell / g.nc[0]) % g.nc[1], cell / (g.nc[0] * g.nc[1])};
  int offs[3][3] = {}, noff[3] = {};
  for (int a = 0; a < 3; a++) {
    noff[a] = 0;
    for (int d = -1; d <= 1; d++) {
      int k = c[a] + d;
      if (g.per[a]) {
        k = ((k % g.nc[a]) + g.nc[a]) % g.nc[a];
      } else if (k < 0 || k >= g.nc[a]) {
        continue;
      }
      bool dup = false;
      for (int q = 0; q < noff[a]; q++) dup |= (offs[a][q] == k);
      if (!dup) offs[a][noff[a]++] = k;
    }
  }
  for (int z = 0; z < noff[2]; z++)
    for (int y = 0; y < noff[1]; y++)
      for (int x = 0; x < noff[0]; x++) {
        int cc = (offs[2][z] * g.nc[1] + offs[1][y]) * g.nc[0] + offs[0][x];
        for (int64_t p = g.cell_start[cc]; p < g.cell_start[cc + 1]; p++) {
          int64_t m = g.order[p];
          if (m != n_atom) out.push_back(m);
        }
      }
  std::sort(out.begin(), out.end());
}

bool all_finite(int64_t n, const double* pos) {
  for (int64_t i = 0; i < 3 * n; i++)
    if (!std::isfinite(pos[i])) return false;
  return true;
}

// ---------------------------------------------------------------------------------
// Half pair list, src/nnlist.jl:23-46: j > n within rcut (PeriodicEuclidean), with
// displacement r = get_displacement(L, X[n], X[m]) = x_n - x_m.
struct PairList {
  std::vector<int64_t> off;
  std::vector<int32_t> j;
  std::vector<double> r;
};

void half_list(int64_t n, const double* pos, const double* L, double rcut, PairList& pl) {
  CellGrid g;
  build_grid(g, n, pos, L, rcut);
  pl.off.assign(n + 1, 0);
  std::vector<std::vector<int32_t>> js(n);
  std::vector<std::vector<double>> rs(n);
#pragma omp parallel
  {
    std::vector<int64_t> cand;
#pragma omp for schedule(dynamic, 64)
    for (int64_t a = 0; a < n; a++) {
      candidates(g, a, cand);
      for (int64_t m : cand) {
        if (m <= a) continue;
        if (pe_dist(L, pos + 3 * a, pos + 3 * m) <= rcut) {
          js[a].push_back((int32_t)m);
          for (int q = 0; q < 3; q++) rs[a].push_back(disp_axis(L[q], pos[3 * a + q], pos[3 * m + q]));
        }
      }
    }
  }
  for (int64_t a = 0; a < n; a++) pl.off[a + 1] = pl.off[a] + (int64_t)js[a].size();
  pl.j.resize(pl.off[n]);
  pl.r.resize(3 * pl.off[n]);
  for (int64_t a = 0; a < n; a++) {
    std::copy(js[a].begin(), js[a].end(), pl.j.begin() + pl.off[a]);
    std::copy(rs[a].begin(), rs[a].end(), pl.r.begin() + 3 * pl.off[a]);
  }
}

// SNAP full list, src/BasisSystems/SNAP/utilities/utl.jl:38-101.  cutsq[ti][tj] =
// ((radii_i + radii_j) * rcutfac)^2 (utl.jl:41-56); candidates within `radius` (cutmax,
// or sqrt(cutmax) when the utl.jl:81 literal radius is requested); rr = x_nb - x_n
// (utl.jl:87); kept when nb != n and rsq <= cutsq (utl.jl:88-89).  Species of both
// atoms index cutsq by their position in snap.species (intended reading of utl.jl:80,86).
void snap_list(int64_t n, const double* pos, const double* L, const int32_t* species, int nsp,
               const double* radii, double rcutfac, int literal_sqrt, PairList& pl) {
  std::vector<double> cutsq(nsp * nsp);
  double cutmax = 0.0;
  for (int a = 0; a < nsp; a++) {
    double cut = 2.0 * radii[a] * rcutfac;
    if (cut > cutmax) cutmax = cut;
    cutsq[a * nsp + a] = cut * cut;
    for (int b = a + 1; b < nsp; b++) {
      double c2 = (radii[a] + radii[b]) * rcutfac;
      cutsq[a * nsp + b] = c2 * c2;
      cutsq[b * nsp + a] = c2 * c2;
    }
  }
  double radius = literal_sqrt ? std::sqrt(cutmax) : cutmax;
  CellGrid g;
  build_grid(g, n, pos, L, radius);
  pl.off.assign(n + 1, 0);
  std::vector<std::vector<int32_t>> js(n);
  std::vector<std::vector<double>> rs(n);
#pragma omp parallel
  {
    std::vector<int64_t> cand;
#pragma omp for schedule(dynamic, 64)
    for (int64_t a = 0; a < n; a++) {
      candidates(g, a, cand);
      for (int64_t m : cand) {
        if (pe_dist(L, pos + 3 * a, pos + 3 * m) > radius) continue;
        double rr[3];
        for (int q = 0; q < 3; q++) rr[q] = -disp_axis(L[q], pos[3 * a + q], pos[3 * m + q]);
        double rsq = rr[0] * rr[0];
        rsq = rsq + rr[1] * rr[1];
        rsq = rsq + rr[2] * rr[2];
        if (rsq <= cutsq[species[a] * nsp + species[m]]) {
          js[a].push_back((int32_t)m);
          for (int q = 0; q < 3; q++) rs[a].push_back(rr[q]);
        }
      }
    }
  }
  for (int64_t a = 0; a < n; a++) pl.off[a + 1] = pl.off[a] + (int64_t)js[a].size();
  pl.j.resize(pl.off[n]);
  pl.r.resize(3 * pl.off[n]);
  for (int64_t a = 0; a < n; a++) {
    std::copy(js[a].begin(), js[a].end(), pl.j.begin() + pl.off[a]);
    std::copy(rs[a].begin(), rs[a].end(), pl.r.begin() + 3 * pl.off[a]);
  }
}

// ---------------------------------------------------------------------------------
// Pair terms (kinds match include/ipg.h).  Formulas are the reference's, literally.
enum { K_LJ = 1, K_BM = 2, K_COUL = 3, K_MORSE = 4, K_ZBL = 5, K_MOCK_R2 = 6 };

// Returns V(R) and g(R) with force f = g(R) * r.
inline void pair_term(int kind, const double* p, double R, double& V, double& g) {
  switch (kind) {
    case K_LJ: {  // src/empirical/lj.jl:35-36 (p = eps, sigma)
      double s = p[1] / R;
      double s6 = std::pow(s, 6), s12 = std::pow(s, 12);
      V = 4.0 * p[0] * (s12 - s6);
      g = 24.0 * p[0] * (2.0 * s12 - s6) / (R * R);
      break;
    }
    case K_BM: {  // src/empirical/bm.jl:38-39 (p = A, rho, sigma, C, D)
      double ex = p[0] * std::exp((p[2] - R) / p[1]);
      double c6 = std::pow(p[3] / R, 6), d8 = std::pow(p[4] / R, 8);
      V = ex + c6 - d8;
      g = ex / (p[1] * R) + (c6 - d8) / (R * R);
      break;
    }
    case K_COUL: {  // src/empirical/coulomb.jl:36-37 (p = q1, q2), k_e = 1 (constants.jl:7)
      double k = 1.0 * p[0] * p[1];
      V = k / R;
      g = k / (R * R * R);
      break;
    }
    case K_MORSE: {  // src/empirical/morse.jl:36-39 (p = D, alpha, sigma)
      double e = std::exp(-p[1] * (R - p[2]));
      V = p[0] * (1.0 - e) * (1.0 - e);
      g = 2.0 * p[0] * p[1] * (1.0 - e) * e / R;
      break;
    }
    case K_ZBL: {  // src/empirical/zbl.jl:27-36 (p = Z1, Z2, e)
      static const double c[4] = {0.18175, 0.50986, 0.28022, 0.02817};
      static const double a[4] = {3.19980, 0.94229, 0.40290, 0.20162};
      double Z1 = p[0], Z2 = p[1], e = p[2];
      double coeff = 1.0 * Z1 * Z2 * e * e;
      double d = R / (0.8854 * 0.529 / (std::pow(Z1, 0.23) + std::pow(Z2, 0.23)));
      double phi = 0.0, dphi = 0.0;
      for (int k = 0; k < 4; k++) {
        double t = std::pow(e, -a[k] * d);
        phi += c[k] * t;
        dphi += a[k] * c[k] * t;
      }
      dphi = -dphi;
      V = coeff * phi / R;
      g = coeff * (phi + d * dphi) / (R * R * R);
      break;
    }
    case K_MOCK_R2: {  // test/mocks.jl:29-34 (p = seed)
      V = R * R * p[0];
      g = R * R * p[0];
      break;
    }
    default:
      V = 0.0;
      g = 0.0;
  }
}

// ---------------------------------------------------------------------------------
// SNAP prebuilt tables: src/BasisSystems/SNAP/types/prebuilt_arrays.jl:48-321.
struct ZIdx {
  int j1, j2, j, ma1min, ma2max, mb1min, mb2max, na, nb, jju;
};

struct Snap {
  int J, nsp;
  double rcutfac, rmin0, rfac0;
  std::vector<double> radii, weight;
  int bzero_flag, bnorm_flag, switch_flag, literal_sqrt;
  int chem_flag = 0, wselfall_flag = 0, literal_chem_z = 0, quadratic_flag = 0;
  int nelem = 1;  // elements resolved by the descriptors: nsp with chem_flag, else 1
  // linear components per species block (get_num_snap_coeffs, utl.jl:8-25), and with the
  // quadratic products B_k B_l (k <= l) appended (LAMMPS_SNAP/snap.jl:45-47)
  int nlin() const { return idxb_max * nelem * nelem * nelem; }
  int ncoef() const { return quadratic_flag ? nlin() + nlin() * (nlin() + 1) / 2 : nlin(); }
  int idxcg_max, idxu_max, idxb_max, idxz_max;
  std::vector<int> idxcg_block, idxu_block, idxb_block, idxz_block;  // [(J+1)^3], [J+1]
  std::vector<int> idxb;                                            // 3 per jjb
  std::vector<ZIdx> idxz;
  std::vector<double> cglist, rootpq, bzero;
  double wself = 1.0;
  int blk(int j1, int j2, int j) const { return (j1 * (J + 1) + j2) * (J + 1) + j; }
  double rpq(int p, int q) const { return rootpq[p * (J + 2) + q]; }
};

// Julia factorial(::Int) products are exact Int64 for twojmax <= 8; long double keeps
// them exact there and avoids the Int64 overflow the reference would hit beyond.
long double factorial_i(int n) {
  long double f = 1.0L;
  for (int k = 2; k <= n; k++) f *= k;
  return f;
}

// prebuilt_arrays.jl:250-257
double deltacg(int j1, int j2, int j) {
  long double sfaccg = factorial_i((j1 + j2 + j) / 2 + 1);
  long double num = factorial_i((j1 + j2 - j) / 2) * factorial_i((j1 - j2 + j) / 2) * factorial_i((-j1 + j2 + j) / 2);
  return std::sqrt((double)num / (double)sfaccg);
}

// Julia integer division `÷` truncates toward zero, like C.
void init_tables(Snap& s) {
  int J = s.J, jd = J + 1;
  s.idxcg_block.assign(jd * jd * jd, 0);
  s.idxu_block.assign(jd, 0);
  s.idxb_block.assign(jd * jd * jd, 0);
  s.idxz_block.assign(jd * jd * jd, 0);
  // bzero: prebuilt_arrays.jl:52-63
  s.bzero.assign(jd, 0.0);
  if (s.bzero_flag) {
    double www = s.wself * s.wself * s.wself;
    for (int j = 0; j <= J; j++) s.bzero[j] = s.bnorm_flag ? www : www * (j + 1);
  }
  int cnt = 0;  // :76-91
  for (int j1 = 0; j1 <= J; j1++)
    for (int j2 = 0; j2 <= j1; j2++)
      for (int j = j1 - j2; j <= std::min(J, j1 + j2); j += 2) {
        s.idxcg_block[s.blk(j1, j2, j)] = cnt;
        cnt += (j1 + 1) * (j2 + 1);
      }
  s.idxcg_max = cnt;
  cnt = 0;  // :95-106
  for (int j = 0; j <= J; j++) {
    s.idxu_block[j] = cnt;
    cnt += (j + 1) * (j + 1);
  }
  s.idxu_max = cnt;
  s.idxb.clear();  // :110-156
  for (int j1 = 0; j1 <= J; j1++)
    for (int j2 = 0; j2 <= j1; j2++)
      for (int j = j1 - j2; j <= std::min(J, j1 + j2); j += 2)
        if (j >= j1) {
          s.idxb_block[s.blk(j1, j2, j)] = (int)s.idxb.size() / 3;
          s.idxb.push_back(j1);
          s.idxb.push_back(j2);
          s.idxb.push_back(j);
        }
  s.idxb_max = (int)s.idxb.size() / 3;
  s.idxz.clear();  // :159-216
  for (int j1 = 0; j1 <= J; j1++)
    for (int j2 = 0; j2 <= j1; j2++)
      for (int j = j1 - j2; j <= std::min(J, j1 + j2); j += 2) {
        s.idxz_block[s.blk(j1, j2, j)] = (int)s.idxz.size();
        for (int mb = 0; 2 * mb <= j; mb++)
          for (int ma = 0; ma <= j; ma++) {
            ZIdx z;
            z.j1 = j1;
            z.j2 = j2;
            z.j = j;
            z.ma1min = std::max(0, (2 * ma - j - j2 + j1) / 2);
            z.ma2max = (2 * ma - j - (2 * z.ma1min - j1) + j2) / 2;
            z.na = std::min(j1, (2 * ma - j + j2 + j1) / 2) - z.ma1min + 1;
            z.mb1min = std::max(0, (2 * mb - j - j2 + j1) / 2);
            z.mb2max = (2 * mb - j - (2 * z.mb1min - j1) + j2) / 2;
            z.nb = std::min(j1, (2 * mb - j + j2 + j1) / 2) - z.mb1min + 1;
            z.jju = s.idxu_block[j] + (j + 1) * mb + ma;
            s.idxz.push_back(z);
          }
      }
  s.idxz_max = (int)s.idxz.size();
  // rootpq: :314-321, rootpq[p][q] = sqrt(p/q) for p,q in 1..J
  s.rootpq.assign((J + 2) * (J + 2), 0.0);
  for (int p = 1; p <= J; p++)
    for (int q = 1; q <= J; q++) s.rootpq[p * (J + 2) + q] = std::sqrt((double)p / (double)q);
  // Clebsch-Gordan: :259-312
  s.cglist.assign(s.idxcg_max, 0.0);
  int idx = 0;
  for (int j1 = 0; j1 <= J; j1++)
    for (int j2 = 0; j2 <= j1; j2++)
      for (int j = j1 - j2; j <= std::min(J, j1 + j2); j += 2)
        for (int m1 = 0; m1 <= j1; m1++) {
          int aa2 = 2 * m1 - j1;
          for (int m2 = 0; m2 <= j2; m2++) {
            int bb2 = 2 * m2 - j2;
            int m = (aa2 + bb2 + j) / 2;
            if (m < 0 || m > j) {
              s.cglist[idx++] = 0.0;
              continue;
            }
            double sum = 0.0;
            int min_z = std::max(0, std::max(-(j - j2 + aa2) / 2, -(j - j1 - bb2) / 2));
            int max_z = std::min((j1 + j2 - j) / 2, std::min((j1 - aa2) / 2, (j2 + bb2) / 2));
            for (int z = min_z; z <= max_z; z++) {
              double ifac = (z % 2 == 0) ? 1.0 : -1.0;
              long double den = factorial_i(z) * factorial_i((j1 + j2 - j) / 2 - z) * factorial_i((j1 - aa2) / 2 - z) *
                            factorial_i((j2 + bb2) / 2 - z) * factorial_i((j - j2 + aa2) / 2 + z) *
                            factorial_i((j - j1 - bb2) / 2 + z);
              sum += ifac / (double)den;
            }
            int cc2 = 2 * m - j;
            double dcg = deltacg(j1, j2, j);
            long double sf = factorial_i((j1 + aa2) / 2) * factorial_i((j1 - aa2) / 2) * factorial_i((j2 + bb2) / 2) *
                         factorial_i((j2 - bb2) / 2) * factorial_i((j + cc2) / 2) * factorial_i((j - cc2) / 2) *
                         (long double)(j + 1);
            double sfaccg = std::sqrt((double)sf);
            s.cglist[idx++] = sum * dcg * sfaccg;
          }
        }
}

// compute_ui.jl:350-364
double compute_sfac(const Snap& s, double r, double rcut) {
  if (!s.switch_flag) return 1.0;
  if (r <= s.rmin0) return 1.0;
  if (r > rcut) return 0.0;
  double rcutfac = M_PI / (rcut - s.rmin0);
  return 0.5 * (std::cos((r - s.rmin0) * rcutfac) + 1.0);
}
// compute_ui.jl:366-380 (the `rcut > rcut` branch of :372 is never taken)
double compute_dsfac(const Snap& s, double r, double rcut) {
  if (!s.switch_flag) return 0.0;
  if (r <= s.rmin0) return 0.0;
  double rcutfac = M_PI / (rcut - s.rmin0);
  return -0.5 * (std::sin((r - s.rmin0) * rcutfac) * rcutfac);
}

// compute_ui.jl:50-129 compute_uarray (full matrix, both halves)
void compute_uarray(const Snap& s, double x, double y, double z, double z0, double r, double* ur, double* ui) {
  double r0inv = 1.0 / std::sqrt(r * r + z0 * z0);
  double a_r = r0inv * z0, a_i = -r0inv * z, b_r = r0inv * y, b_i = -r0inv * x;
  ur[0] = 1.0;
  ui[0] = 0.0;
  for (int j = 1; j <= s.J; j++) {
    int jju = s.idxu_block[j], jjup = s.idxu_block[j - 1];
    for (int mb = 0; 2 * mb <= j; mb++) {
      ur[jju] = 0.0;
      ui[jju] = 0.0;
      for (int ma = 0; ma < j; ma++) {
        double rootpq = s.rpq(j - ma, j - mb);
        ur[jju] += rootpq * (a_r * ur[jjup] + a_i * ui[jjup]);
        ui[jju] += rootpq * (a_r * ui[jjup] - a_i * ur[jjup]);
        rootpq = s.rpq(ma + 1, j - mb);
        ur[jju + 1] = -rootpq * (b_r * ur[jjup] + b_i * ui[jjup]);
        ui[jju + 1] = -rootpq * (b_r * ui[jjup] - b_i * ur[jjup]);
        jju++;
        jjup++;
      }
      jju++;
    }
    jju = s.idxu_block[j];
    jjup = jju + (j + 1) * (j + 1) - 1;
    int mbpar = 1;
    for (int mb = 0; 2 * mb <= j; mb++) {
      int mapar = mbpar;
      for (int ma = 0; ma <= j; ma++) {
        if (mapar == 1) {
          ur[jjup] = ur[jju];
          ui[jjup] = -ui[jju];
        } else {
          ur[jjup] = -ur[jju];
          ui[jjup] = ui[jju];
        }
        mapar = -mapar;
        jju++;
        jjup--;
      }
      mbpar = -mbpar;
    }
  }
}

// compute_ui.jl:186-326 compute_duarray (+ compute_duidrj :328-347 prologue)
void compute_duidrj(const Snap& s, const double* rij, double wj, double rcut, const double* ur, const double* ui,
                    double* dur, double* dui /* [idxu_max][3] */) {
  double x = rij[0], y = rij[1], z = rij[2];
  double rsq = x * x + y * y + z * z;
  double r = std::sqrt(rsq);
  double rscale0 = s.rfac0 * M_PI / (rcut - s.rmin0);
  double theta0 = (r - s.rmin0) * rscale0;
  double cs = std::cos(theta0), sn = std::sin(theta0);
  double z0 = r * cs / sn;
  double dz0dr = z0 / r - (r * rscale0) * (rsq + z0 * z0) / rsq;

  double rinv = 1.0 / r;
  double ux = x * rinv, uy = y * rinv, uz = z * rinv;
  double r0inv = 1.0 / std::sqrt(r * r + z0 * z0);
  double a_r = z0 * r0inv, a_i = -z * r0inv, b_r = y * r0inv, b_i = -x * r0inv;
  double dr0invdr = -r0inv * r0inv * r0inv * (r + z0 * dz0dr);
  double dr0inv[3] = {dr0invdr * ux, dr0invdr * uy, dr0invdr * uz};
  double dz0[3] = {dz0dr * ux, dz0dr * uy, dz0dr * uz};
  double da_r[3], da_i[3], db_r[3], db_i[3];
  for (int k = 0; k < 3; k++) {
    da_r[k] = dz0[k] * r0inv + z0 * dr0inv[k];
    da_i[k] = -z * dr0inv[k];
    db_r[k] = y * dr0inv[k];
    db_i[k] = -x * dr0inv[k];
  }
  da_i[2] += -r0inv;
  db_i[0] += -r0inv;
  db_r[1] += r0inv;

  for (int k = 0; k < 3; k++) {
    dur[k] = 0.0;
    dui[k] = 0.0;
  }
  for (int j = 1; j <= s.J; j++) {
    int jju = s.idxu_block[j], jjup = s.idxu_block[j - 1];
    for (int mb = 0; 2 * mb <= j; mb++) {
      for (int k = 0; k < 3; k++) {
        dur[3 * jju + k] = 0.0;
        dui[3 * jju + k] = 0.0;
      }
      for (int ma = 0; ma < j; ma++) {
        double rootpq = s.rpq(j - ma, j - mb);
        for (int k = 0; k < 3; k++) {
          dur[3 * jju + k] += rootpq * (da_r[k] * ur[jjup] + da_i[k] * ui[jjup] + a_r * dur[3 * jjup + k] +
                                        a_i * dui[3 * jjup + k]);
          dui[3 * jju + k] += rootpq * (da_r[k] * ui[jjup] - da_i[k] * ur[jjup] + a_r * dui[3 * jjup + k] -
                                        a_i * dur[3 * jjup + k]);
        }
        rootpq = s.rpq(ma + 1, j - mb);
        for (int k = 0; k < 3; k++) {
          dur[3 * (jju + 1) + k] = -rootpq * (db_r[k] * ur[jjup] + db_i[k] * ui[jjup] + b_r * dur[3 * jjup + k] +
                                              b_i * dui[3 * jjup + k]);
          dui[3 * (jju + 1) + k] = -rootpq * (db_r[k] * ui[jjup] - db_i[k] * ur[jjup] + b_r * dui[3 * jjup + k] -
                                              b_i * dur[3 * jjup + k]);
        }
        jju++;
        jjup++;
      }
      jju++;
    }
    jju = s.idxu_block[j];
    jjup = jju + (j + 1) * (j + 1) - 1;
    int mbpar = 1;
    for (int mb = 0; 2 * mb <= j; mb++) {
      int mapar = mbpar;
      for (int ma = 0; ma <= j; ma++) {
        for (int k = 0; k < 3; k++) {
          if (mapar == 1) {
            dur[3 * jjup + k] = dur[3 * jju + k];
            dui[3 * jjup + k] = -dui[3 * jju + k];
          } else {
            dur[3 * jjup + k] = -dur[3 * jju + k];
            dui[3 * jjup + k] = dui[3 * jju + k];
          }
        }
        mapar = -mapar;
        jju++;
        jjup--;
      }
      mbpar = -mbpar;
    }
  }
  double sfac = compute_sfac(s, r, rcut) * wj;
  double dsfac = compute_dsfac(s, r, rcut) * wj;
  double u3[3] = {ux, uy, uz};
  for (int j = 0; j <= s.J; j++) {
    int jju = s.idxu_block[j];
    for (int mb = 0; 2 * mb <= j; mb++)
      for (int ma = 0; ma <= j; ma++) {
        for (int k = 0; k < 3; k++) {
          dur[3 * jju + k] = dsfac * ur[jju] * u3[k] + sfac * dur[3 * jju + k];
          dui[3 * jju + k] = dsfac * ui[jju] * u3[k] + sfac * dui[3 * jju + k];
        }
        jju++;
      }
  }
}

// Per-atom state of compute_all_descriptors (snap.jl:251-310).
struct AtomWork {
  std::vector<double> utr, uti;  // Utot [nelem][idxu_max]
  std::vector<double> ulr, uli;  // per-neighbor U [nnbr][idxu_max]
  std::vector<double> zr, zi;    // Z [nelem^2][idxz_max]
  std::vector<double> yr, yi;    // Y [idxu_max] (adjoint restatement)
  std::vector<double> b;         // B [nlin]
  std::vector<double> dur, dui;  // dU [idxu_max][3]
  std::vector<double> db;        // dB [nlin][3]
};

// compute_ui.jl:5-44, 131-175: Utot for atom i from its neighbor rows; with chem_flag one
// Utot per element (the neighbor's element, add_uarraytot :155-175), wself on the diagonal of
// the centre's element or, with wselfall_flag, of every element (zero_uarraytot :131-152).
void compute_ui(const Snap& s, int64_t nn, const double* r, const int32_t* jn, int32_t si, const int32_t* species,
                AtomWork& w) {
  int U = s.idxu_max;
  w.utr.assign((size_t)s.nelem * U, 0.0);
  w.uti.assign((size_t)s.nelem * U, 0.0);
  const int ielem = s.chem_flag ? si : 0;
  for (int e = 0; e < s.nelem; e++) {
    if (!(e == ielem || s.wselfall_flag)) continue;
    for (int j = 0; j <= s.J; j++) {  // zero_uarraytot: wself on the diagonal
      int jju = s.idxu_block[j];
      for (int mb = 0; mb <= j; mb++)
        for (int ma = 0; ma <= j; ma++) {
          if (ma == mb) w.utr[(size_t)e * U + jju] = s.wself;
          jju++;
        }
    }
  }
  w.ulr.assign((size_t)nn * U, 0.0);
  w.uli.assign((size_t)nn * U, 0.0);
  for (int64_t k = 0; k < nn; k++) {
    int32_t sj = species[jn[k]];
    double rcutij = (s.radii[si] + s.radii[sj]) * s.rcutfac;  // runtime_arrays.jl:50
    double wj = s.weight[sj];
    double x = r[3 * k], y = r[3 * k + 1], z = r[3 * k + 2];
    double rsq = x * x + y * y + z * z;
    double rr = std::sqrt(rsq);
    double theta0 = (rr - s.rmin0) * s.rfac0 * M_PI / (rcutij - s.rmin0);
    double z0 = rr / std::tan(theta0);
    double* ur = &w.ulr[(size_t)k * U];
    double* ui = &w.uli[(size_t)k * U];
    compute_uarray(s, x, y, z, z0, rr, ur, ui);
    double sfac = compute_sfac(s, rr, rcutij) * wj;
    const size_t eo = (size_t)(s.chem_flag ? sj : 0) * U;
    for (int q = 0; q < U; q++) {
      w.utr[eo + q] += sfac * ur[q];
      w.uti[eo + q] += sfac * ui[q];
    }
  }
}

// compute_z.jl:1-62: Z of every ordered element pair (elem1, elem2), idouble = elem1*nelem
// + elem2, at Z[idouble*idxz_max + jjz].  literal_chem_z reproduces the reference's indexing
// (:19-20 zero the slot idouble*idxz_max + jjz, :44-47 accumulate into and divide slot jjz):
// every pair then sums into the first block, dividing the running sum by j+1 after each pair
// when bnorm_flag is set, and the other blocks stay zero.
void compute_zi(const Snap& s, AtomWork& w) {
  const int M = s.idxz_max, U = s.idxu_max;
  w.zr.assign((size_t)s.nelem * s.nelem * M, 0.0);
  w.zi.assign((size_t)s.nelem * s.nelem * M, 0.0);
  int idouble = 0;
  for (int e1 = 0; e1 < s.nelem; e1++)
    for (int e2 = 0; e2 < s.nelem; e2++) {
      const double* u1r = &w.utr[(size_t)e1 * U];
      const double* u1i = &w.uti[(size_t)e1 * U];
      const double* u2r = &w.utr[(size_t)e2 * U];
      const double* u2i = &w.uti[(size_t)e2 * U];
      for (int jjz = 0; jjz < M; jjz++) {
        const ZIdx& q = s.idxz[jjz];
        const double* cgblock = &s.cglist[s.idxcg_block[s.blk(q.j1, q.j2, q.j)]];
        const size_t zslot = s.literal_chem_z ? (size_t)jjz : (size_t)idouble * M + jjz;
        w.zr[(size_t)idouble * M + jjz] = 0.0;
        w.zi[(size_t)idouble * M + jjz] = 0.0;
        double zr = w.zr[zslot], zi = w.zi[zslot];
        int jju1 = s.idxu_block[q.j1] + (q.j1 + 1) * q.mb1min;
        int jju2 = s.idxu_block[q.j2] + (q.j2 + 1) * q.mb2max;
        int icgb = q.mb1min * (q.j2 + 1) + q.mb2max;
        for (int ib = 0; ib < q.nb; ib++) {
          double sr = 0.0, si = 0.0;
          int ma1 = q.ma1min, ma2 = q.ma2max;
          int icga = q.ma1min * (q.j2 + 1) + q.ma2max;
          for (int ia = 0; ia < q.na; ia++) {
            double a1r = u1r[jju1 + ma1], a1i = u1i[jju1 + ma1];
            double a2r = u2r[jju2 + ma2], a2i = u2i[jju2 + ma2];
            sr += cgblock[icga] * (a1r * a2r - a1i * a2i);
            si += cgblock[icga] * (a1r * a2i + a1i * a2r);
            ma1++;
            ma2--;
            icga += q.j2;
          }
          zr += cgblock[icgb] * sr;
          zi += cgblock[icgb] * si;
          jju1 += q.j1 + 1;
          jju2 -= q.j2 + 1;
          icgb += q.j2;
        }
        if (s.bnorm_flag) {
          zr /= (q.j + 1);
          zi /= (q.j + 1);
        }
        w.zr[zslot] = zr;
        w.zi[zslot] = zi;
      }
      idouble++;
    }
}

// compute_b.jl:5-95: B of every element triple (elem1, elem2, elem3), itriple =
// (elem1*nelem + elem2)*nelem + elem3, at B[itriple*idxb_max + jjb]: Utot of elem3 against Z of
// (elem1, elem2).  bzero: the centre element's triple (ielem, ielem, ielem), or every triple with
// wselfall_flag, as LAMMPS' compute_bi(ielem).  (The reference wraps the whole computation in a
// loop over ielem that recomputes B each time, so only the last element's triple would keep its
// shift; the per-centre shift is taken here.)
void compute_bi(const Snap& s, AtomWork& w, int32_t si) {
  const int K = s.idxb_max, U = s.idxu_max, M = s.idxz_max, n = s.nelem;
  w.b.assign((size_t)s.nlin(), 0.0);
  int itriple = 0;
  for (int e1 = 0; e1 < n; e1++)
    for (int e2 = 0; e2 < n; e2++) {
      const size_t zo = (size_t)(e1 * n + e2) * M;
      for (int e3 = 0; e3 < n; e3++) {
        const double* ur = &w.utr[(size_t)e3 * U];
        const double* ui = &w.uti[(size_t)e3 * U];
        for (int jjb = 0; jjb < K; jjb++) {
          int j1 = s.idxb[3 * jjb], j2 = s.idxb[3 * jjb + 1], j = s.idxb[3 * jjb + 2];
          size_t jjz = zo + s.idxz_block[s.blk(j1, j2, j)];
          int jju = s.idxu_block[j];
          double sumzu = 0.0;
          for (int mb = 0; 2 * mb < j; mb++)
            for (int ma = 0; ma <= j; ma++) {
              sumzu += ur[jju] * w.zr[jjz] + ui[jju] * w.zi[jjz];
              jjz++;
              jju++;
            }
          if (j % 2 == 0) {
            int mb = j / 2;
            for (int ma = 0; ma < mb; ma++) {
              sumzu += ur[jju] * w.zr[jjz] + ui[jju] * w.zi[jjz];
              jjz++;
              jju++;
            }
            sumzu += 0.5 * (ur[jju] * w.zr[jjz] + ui[jju] * w.zi[jjz]);
          }
          w.b[(size_t)itriple * K + jjb] = 2.0 * sumzu;
        }
        itriple++;
      }
    }
  if (s.bzero_flag) {
    const int ielem = s.chem_flag ? si : 0;
    for (int t = 0; t < n * n * n; t++) {
      if (!s.wselfall_flag && t != (ielem * n + ielem) * n + ielem) continue;
      for (int jjb = 0; jjb < K; jjb++) w.b[(size_t)t * K + jjb] -= s.bzero[s.idxb[3 * jjb + 2]];
    }
  }
}

// Half-plane sum of Re(conj(du[:,k]) * z) over level j starting at Z index jjz
// (the inner loops of compute_b.jl:225-266).
inline void sum_half(const Snap& s, const AtomWork& w, int j, size_t jjz, double* out3) {
  int jju = s.idxu_block[j];
  double acc[3] = {0.0, 0.0, 0.0};
  for (int mb = 0; 2 * mb < j; mb++)
    for (int ma = 0; ma <= j; ma++) {
      for (int k = 0; k < 3; k++) acc[k] += w.dur[3 * jju + k] * w.zr[jjz] + w.dui[3 * jju + k] * w.zi[jjz];
      jjz++;
      jju++;
    }
  if (j % 2 == 0) {
    int mb = j / 2;
    for (int ma = 0; ma < mb; ma++) {
      for (int k = 0; k < 3; k++) acc[k] += w.dur[3 * jju + k] * w.zr[jjz] + w.dui[3 * jju + k] * w.zi[jjz];
      jjz++;
      jju++;
    }
    for (int k = 0; k < 3; k++) acc[k] += (w.dur[3 * jju + k] * w.zr[jjz] + w.dui[3 * jju + k] * w.zi[jjz]) * 0.5;
  }
  for (int k = 0; k < 3; k++) out3[k] = acc[k];
}

// compute_b.jl:104-342 compute_dbidrj for a neighbor of element jelem (elem3 = jelem with
// chem_flag, else 0): for every element pair, the three terms of each component land in their
// own triples (:196, :250, :305).
void compute_dbidrj(const Snap& s, AtomWork& w, int32_t jelem) {
  const int K = s.idxb_max, M = s.idxz_max, n = s.nelem;
  const int e3 = s.chem_flag ? jelem : 0;
  w.db.assign((size_t)s.nlin() * 3, 0.0);
  for (int jjb = 0; jjb < K; jjb++) {
    int j1 = s.idxb[3 * jjb], j2 = s.idxb[3 * jjb + 1], j = s.idxb[3 * jjb + 2];
    for (int e1 = 0; e1 < n; e1++)
      for (int e2 = 0; e2 < n; e2++) {
        double t[3];
        size_t it = (size_t)((e1 * n + e2) * n + e3);
        sum_half(s, w, j, (size_t)(e1 * n + e2) * M + s.idxz_block[s.blk(j1, j2, j)], t);
        for (int k = 0; k < 3; k++) w.db[3 * (it * K + jjb) + k] = 2.0 * t[k];
        double j1fac = (j + 1) / (j1 + 1.0);
        it = (size_t)((e3 * n + e2) * n + e1);
        sum_half(s, w, j1, (size_t)(e1 * n + e2) * M + s.idxz_block[s.blk(j, j2, j1)], t);
        for (int k = 0; k < 3; k++) w.db[3 * (it * K + jjb) + k] += s.bnorm_flag ? 2.0 * t[k] : 2.0 * t[k] * j1fac;
        double j2fac = (j + 1) / (j2 + 1.0);
        it = (size_t)((e1 * n + e3) * n + e2);
        sum_half(s, w, j2, (size_t)(e2 * n + e1) * M + s.idxz_block[s.blk(j, j1, j2)], t);
        for (int k = 0; k < 3; k++) w.db[3 * (it * K + jjb) + k] += s.bnorm_flag ? 2.0 * t[k] : 2.0 * t[k] * j2fac;
      }
  }
}

// Quadratic SNAP (the quadratic option of LAMMPS_SNAP/snap.jl:45-47, LAMMPS' layout): the
// linear components b [nlin] are followed by 0.5 b_k b_k and b_k b_l (l > k), k outer.
void quad_extend(const Snap& s, const double* b, double* out) {
  const int K = s.nlin();
  std::memcpy(out, b, sizeof(double) * K);
  size_t q = K;
  for (int k = 0; k < K; k++) {
    out[q++] = 0.5 * b[k] * b[k];
    for (int l = k + 1; l < K; l++) out[q++] = b[k] * b[l];
  }
}
// Their derivative for one pair: d(0.5 b_k^2) = b_k db_k, d(b_k b_l) = b_l db_k + b_k db_l.
void quad_extend_d(const Snap& s, const double* b, const double* db, double* out) {
  const int K = s.nlin();
  std::memcpy(out, db, sizeof(double) * 3 * K);
  size_t q = K;
  for (int k = 0; k < K; k++) {
    for (int c = 0; c < 3; c++) out[3 * q + c] = b[k] * db[3 * k + c];
    q++;
    for (int l = k + 1; l < K; l++) {
      for (int c = 0; c < 3; c++) out[3 * q + c] = b[l] * db[3 * k + c] + b[k] * db[3 * l + c];
      q++;
    }
  }
}
// The linear coefficients that give the same forces: beta_eff[k] = beta[k] + sum_l a_kl b_l with
// a the symmetric matrix of the quadratic coefficients (a_kk from 0.5 b_k^2).
void quad_beta_eff(const Snap& s, const double* beta, const double* b, double* out) {
  const int K = s.nlin();
  for (int k = 0; k < K; k++) out[k] = beta[k];
  size_t q = K;
  for (int k = 0; k < K; k++) {
    out[k] += beta[q++] * b[k];
    for (int l = k + 1; l < K; l++) {
      out[k] += beta[q] * b[l];
      out[l] += beta[q] * b[k];
      q++;
    }
  }
}

// Adjoint restatement.  Y follows the design of compute_yi.jl:6-122 (multiplicity 3/2/1
// and the (j1+1)/(j+1) factor), written from the derivative of beta.B with respect to
// U; the reference file itself does not run (undefined names at :8,14,90,108,113).
void compute_yi(const Snap& s, const double* beta, AtomWork& w) {
  w.yr.assign(s.idxu_max, 0.0);
  w.yi.assign(s.idxu_max, 0.0);
  for (int jjz = 0; jjz < s.idxz_max; jjz++) {
    const ZIdx& q = s.idxz[jjz];
    int j1 = q.j1, j2 = q.j2, j = q.j;
    double betaj;
    if (j >= j1) {
      int jjb = s.idxb_block[s.blk(j1, j2, j)];
      if (j1 == j) betaj = (j2 == j) ? 3.0 * beta[jjb] : 2.0 * beta[jjb];
      else betaj = beta[jjb];
    } else if (j >= j2) {
      int jjb = s.idxb_block[s.blk(j, j2, j1)];
      betaj = (j2 == j) ? 2.0 * beta[jjb] : beta[jjb];
    } else {
      int jjb = s.idxb_block[s.blk(j2, j, j1)];
      betaj = beta[jjb];
    }
    if (!s.bnorm_flag && j1 > j) betaj *= (j1 + 1) / (j + 1.0);
    w.yr[q.jju] += betaj * w.zr[jjz];
    w.yi[q.jju] += betaj * w.zi[jjz];
  }
}

// compute_dij.jl:5-74 design: dE_i/dr_ij = 2 sum_half Re(conj(dU) Y), middle column 1/2.
void compute_deidrj(const Snap& s, const AtomWork& w, double* dedr) {
  double acc[3] = {0.0, 0.0, 0.0};
  for (int j = 0; j <= s.J; j++) {
    int jju = s.idxu_block[j];
    for (int mb = 0; 2 * mb < j; mb++)
      for (int ma = 0; ma <= j; ma++) {
        for (int k = 0; k < 3; k++) acc[k] += w.dur[3 * jju + k] * w.yr[jju] + w.dui[3 * jju + k] * w.yi[jju];
        jju++;
      }
    if (j % 2 == 0) {
      int mb = j / 2;
      for (int ma = 0; ma < mb; ma++) {
        for (int k = 0; k < 3; k++) acc[k] += w.dur[3 * jju + k] * w.yr[jju] + w.dui[3 * jju + k] * w.yi[jju];
        jju++;
      }
      for (int k = 0; k < 3; k++) acc[k] += (w.dur[3 * jju + k] * w.yr[jju] + w.dui[3 * jju + k] * w.yi[jju]) * 0.5;
    }
  }
  for (int k = 0; k < 3; k++) dedr[k] = 2.0 * acc[k];
}

int snap_check(const Snap& s, int64_t n, const double* pos, const int32_t* species, const double* L) {
  if (n < 0) return -1;
  if (!all_finite(n, pos)) return -6;
  for (int64_t i = 0; i < n; i++)
    if (species[i] < 0 || species[i] >= s.nsp) return -7;
  for (int a = 0; a < 3; a++)
    if (!(L[a] > 0.0)) return -1;
  return 0;
}

}  // namespace

extern "C" {

// ----- neighbor lists -------------------------------------------------------------
// Returns the number of pairs, or a negative status.  When cap >= npairs the arrays are
// filled: offsets [n+1], j [npairs] (0-based), r [3*npairs].
int64_t orc_nlist_half(int64_t n, const double* pos, const double* L, double rcut, int64_t* offsets, int32_t* j,
                       double* r, int64_t cap) {
  if (!all_finite(n, pos)) return -6;
  PairList pl;
  half_list(n, pos, L, rcut, pl);
  int64_t np = pl.off[n];
  if (offsets && j && r && cap >= np) {
    std::memcpy(offsets, pl.off.data(), sizeof(int64_t) * (n + 1));
    std::memcpy(j, pl.j.data(), sizeof(int32_t) * np);
    std::memcpy(r, pl.r.data(), sizeof(double) * 3 * np);
  }
  return np;
}

int64_t orc_nlist_snap(int64_t n, const double* pos, const double* L, const int32_t* species, int32_t nsp,
                       const double* radii, double rcutfac, int32_t literal_sqrt, int64_t* offsets, int32_t* j,
                       double* r, int64_t cap) {
  if (!all_finite(n, pos)) return -6;
  PairList pl;
  snap_list(n, pos, L, species, nsp, radii, rcutfac, literal_sqrt, pl);
  int64_t np = pl.off[n];
  if (offsets && j && r && cap >= np) {
    std::memcpy(offsets, pl.off.data(), sizeof(int64_t) * (n + 1));
    std::memcpy(j, pl.j.data(), sizeof(int32_t) * np);
    std::memcpy(r, pl.r.data(), sizeof(double) * 3 * np);
  }
  return np;
}

// ----- pair potentials --------------------------------------------------------------
// One term = one EmpiricalPotential; the LinearCombinationPotential sum
// (src/mixed/linear_combination_potential.jl:27-39) is sum_t coeff_t * term_t, and each
// term runs _perform_pairwise (src/types/empirical_potential.jl:20-67) with its own
// neighbor list at its own cutoff and its own species filter.
int orc_pair_eval(int64_t n, const double* pos, const int32_t* species, const double* L, int32_t nterms,
                  const int32_t* kinds, const double* coeffs, const double* rcuts, const uint64_t* masks,
                  const double* params, double* E, double* F, double* W6) {
  if (!all_finite(n, pos)) return -6;
  for (int64_t i = 0; i < n; i++)
    if (species[i] < 0 || species[i] >= 64) return -7;
  double Etot = 0.0, Wtot[6] = {0, 0, 0, 0, 0, 0};
  std::vector<double> Ftot(3 * n, 0.0);
  for (int t = 0; t < nterms; t++) {
    PairList pl;
    half_list(n, pos, L, rcuts[t], pl);
    const double* p = params + 8 * t;
    uint64_t mask = masks[t];
    double e = 0.0, w[6] = {0, 0, 0, 0, 0, 0};
    std::vector<double> f(3 * n, 0.0);
    for (int64_t a = 0; a < n; a++) {
      if (!((mask >> species[a]) & 1ull)) continue;
      for (int64_t q = pl.off[a]; q < pl.off[a + 1]; q++) {
        int32_t m = pl.j[q];
        if (!((mask >> species[m]) & 1ull)) continue;
        const double* r = &pl.r[3 * q];
        double R = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        double V, g;
        pair_term(kinds[t], p, R, V, g);
        e += V;
        double fo[3] = {g * r[0], g * r[1], g * r[2]};
        for (int k = 0; k < 3; k++) {
          f[3 * a + k] += fo[k];
          f[3 * m + k] -= fo[k];
        }
        // empirical_potential.jl:63-64: r * f' -> [xx, yy, zz, zy, zx, yx]
        w[0] += r[0] * fo[0];
        w[1] += r[1] * fo[1];
        w[2] += r[2] * fo[2];
        w[3] += r[2] * fo[1];
        w[4] += r[2] * fo[0];
        w[5] += r[1] * fo[0];
      }
    }
    Etot += coeffs[t] * e;
    for (int64_t k = 0; k < 3 * n; k++) Ftot[k] += coeffs[t] * f[k];
    for (int k = 0; k < 6; k++) Wtot[k] += coeffs[t] * w[k];
  }
  if (E) *E = Etot;
  if (F) std::memcpy(F, Ftot.data(), sizeof(double) * 3 * n);
  if (W6) std::memcpy(W6, Wtot, sizeof(double) * 6);
  return 0;
}

// ----- SNAP -------------------------------------------------------------------------
void* orc_snap_create(int32_t twojmax, int32_t nsp, double rcutfac, double rmin0, double rfac0, const double* radii,
                      const double* weight, int32_t bzero_flag, int32_t bnorm_flag, int32_t switch_flag,
                      int32_t literal_sqrt, int32_t chem_flag, int32_t wselfall_flag, int32_t literal_chem_z,
                      int32_t quadratic_flag) {
  if (twojmax < 0 || twojmax > 14 || nsp < 1 || nsp > 64) return nullptr;
  Snap* s = new Snap();
  s->J = twojmax;
  s->nsp = nsp;
  s->rcutfac = rcutfac;
  s->rmin0 = rmin0;
  s->rfac0 = rfac0;
  s->radii.assign(radii, radii + nsp);
  s->weight.assign(weight, weight + nsp);
  s->bzero_flag = bzero_flag;
  s->bnorm_flag = bnorm_flag;
  s->switch_flag = switch_flag;
  s->literal_sqrt = literal_sqrt;
  s->chem_flag = chem_flag;
  s->wselfall_flag = wselfall_flag;
  s->literal_chem_z = literal_chem_z;
  s->quadratic_flag = quadratic_flag;
  s->nelem = chem_flag ? nsp : 1;
  init_tables(*s);
  return s;
}

// Components per species block: get_num_snap_coeffs (utl.jl:8-25), with the quadratic products.
int32_t orc_snap_ncoef(void* h) { return static_cast<Snap*>(h)->ncoef(); }

void orc_snap_destroy(void* h) { delete static_cast<Snap*>(h); }

// sizes: [idxu_max, idxz_max, idxb_max, idxcg_max]
void orc_snap_sizes(void* h, int32_t* out4) {
  Snap* s = static_cast<Snap*>(h);
  out4[0] = s->idxu_max;
  out4[1] = s->idxz_max;
  out4[2] = s->idxb_max;
  out4[3] = s->idxcg_max;
}

void orc_snap_cglist(void* h, double* out) {
  Snap* s = static_cast<Snap*>(h);
  std::memcpy(out, s->cglist.data(), sizeof(double) * s->idxcg_max);
}

// idxz as 10 ints per entry; idxb as 3 ints per entry; idxcg_block/idxz_block (J+1)^3
void orc_snap_index_tables(void* h, int32_t* idxz10, int32_t* idxb3, int32_t* idxcg_block, int32_t* idxz_block,
                           int32_t* idxu_block) {
  Snap* s = static_cast<Snap*>(h);
  for (int k = 0; k < s->idxz_max; k++) {
    const ZIdx& q = s->idxz[k];
    int32_t v[10] = {q.j1, q.j2, q.j, q.ma1min, q.ma2max, q.mb1min, q.mb2max, q.na, q.nb, q.jju};
    std::memcpy(idxz10 + 10 * k, v, sizeof(v));
  }
  for (int k = 0; k < 3 * s->idxb_max; k++) idxb3[k] = s->idxb[k];
  int jd = s->J + 1;
  for (int k = 0; k < jd * jd * jd; k++) {
    idxcg_block[k] = s->idxcg_block[k];
    idxz_block[k] = s->idxz_block[k];
  }
  for (int k = 0; k < jd; k++) idxu_block[k] = s->idxu_block[k];
}

// compute_all_descriptors (snap.jl:251-310): B [n][K], dB [n][K*nsp][3] (Julia 3 x K*nsp
// column-major per atom), W [K*nsp][6] (6 x K*nsp column-major).  Any output may be null.
// Utot per atom may also be exported ([n][idxu_max][2]) for kernel-level checks.
int orc_snap_descriptors(void* h, int64_t n, const double* pos, const int32_t* species, const double* L, double* B,
                         double* dB, double* W, double* utot_out) {
  Snap& s = *static_cast<Snap*>(h);
  int st = snap_check(s, n, pos, species, L);
  if (st) return st;
  PairList pl;
  snap_list(n, pos, L, species, s.nsp, s.radii.data(), s.rcutfac, s.literal_sqrt, pl);
  int K = s.ncoef(), Kn = K * s.nsp;
  if (dB) std::memset(dB, 0, sizeof(double) * (size_t)n * 3 * Kn);
  if (W) std::memset(W, 0, sizeof(double) * 6 * Kn);
  AtomWork w;
  std::vector<double> bx(K), dbx(3 * (size_t)K);
  for (int64_t i = 0; i < n; i++) {
    int64_t nn = pl.off[i + 1] - pl.off[i];
    const double* r = &pl.r[3 * pl.off[i]];
    const int32_t* jn = &pl.j[pl.off[i]];
    int32_t si = species[i];
    compute_ui(s, nn, r, jn, si, species, w);
    if (utot_out)
      for (int q = 0; q < s.idxu_max; q++) {
        utot_out[((size_t)i * s.idxu_max + q) * 2] = w.utr[q];
        utot_out[((size_t)i * s.idxu_max + q) * 2 + 1] = w.uti[q];
      }
    compute_zi(s, w);
    compute_bi(s, w, si);
    if (s.quadratic_flag)
      quad_extend(s, w.b.data(), bx.data());
    else
      bx = w.b;
    if (B) std::memcpy(B + (size_t)i * K, bx.data(), sizeof(double) * K);
    if (!dB && !W) continue;
    int ioff = K * si;
    w.dur.assign((size_t)s.idxu_max * 3, 0.0);
    w.dui.assign((size_t)s.idxu_max * 3, 0.0);
    for (int64_t k = 0; k < nn; k++) {
      int32_t jj = jn[k];
      int32_t sj = species[jj];
      double rcut = (s.radii[si] + s.radii[sj]) * s.rcutfac;
      compute_duidrj(s, r + 3 * k, s.weight[sj], rcut, &w.ulr[(size_t)k * s.idxu_max],
                     &w.uli[(size_t)k * s.idxu_max], w.dur.data(), w.dui.data());
      compute_dbidrj(s, w, sj);
      if (s.quadratic_flag)
        quad_extend_d(s, w.b.data(), w.db.data(), dbx.data());
      else
        dbx = w.db;
      if (dB)
        for (int q = 0; q < K; q++)
          for (int c = 0; c < 3; c++) {
            dB[((size_t)i * Kn + ioff + q) * 3 + c] += dbx[3 * q + c];
            dB[((size_t)jj * Kn + ioff + q) * 3 + c] -= dbx[3 * q + c];
          }
      if (W) {
        const double* xi = pos + 3 * i;
        const double* xj = pos + 3 * jj;
        for (int q = 0; q < K; q++) {
          const double* d = &dbx[3 * q];
          double* wc = W + (size_t)(ioff + q) * 6;
          wc[0] += d[0] * xi[0] - d[0] * xj[0];
          wc[1] += d[1] * xi[1] - d[1] * xj[1];
          wc[2] += d[2] * xi[2] - d[2] * xj[2];
          wc[3] += d[1] * xi[2] - d[1] * xj[2];
          wc[4] += d[0] * xi[2] - d[0] * xj[2];
          wc[5] += d[0] * xi[1] - d[0] * xj[1];
        }
      }
    }
  }
  return 0;
}

// Energy and forces for LBasisPotential over SNAP (linear_potential.jl:20-49 with the
// per-species beta blocks beta[nsp][K]).  mode 0 = plain (dB/dr contracted with beta),
// mode 1 = adjoint (Y, dE/dr).  Only centre atoms in [i0, i1) are evaluated (a bounded
// sample for timing); i0 = 0, i1 = n gives the full result.  W6 is the reference's
// absolute-position virial contracted with beta (snap.jl:292-306).
int orc_snap_energy_forces(void* h, int64_t n, const double* pos, const int32_t* species, const double* L,
                           const double* beta, double beta0, int32_t mode, int64_t i0, int64_t i1, double* E,
                           double* F, double* W6, double* Ei, int32_t nthreads) {
  Snap& s = *static_cast<Snap*>(h);
  int st = snap_check(s, n, pos, species, L);
  if (st) return st;
  if (i0 < 0) i0 = 0;
  if (i1 > n) i1 = n;
  PairList pl;
  snap_list(n, pos, L, species, s.nsp, s.radii.data(), s.rcutfac, s.literal_sqrt, pl);
  int K = s.ncoef(), KL = s.nlin();
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
  int nt = omp_get_max_threads();
#else
  int nt = 1;
#endif
  std::vector<std::vector<double>> Fth(nt, std::vector<double>(F ? 3 * n : 0, 0.0));
  std::vector<double> Eth(nt, 0.0), Wth(6 * nt, 0.0);
#pragma omp parallel
  {
#ifdef _OPENMP
    int tid = omp_get_thread_num();
#else
    int tid = 0;
#endif
    AtomWork w;
    std::vector<double> bx(K), beff(KL);
#pragma omp for schedule(dynamic, 4)
    for (int64_t i = i0; i < i1; i++) {
      int64_t nn = pl.off[i + 1] - pl.off[i];
      const double* r = &pl.r[3 * pl.off[i]];
      const int32_t* jn = &pl.j[pl.off[i]];
      int32_t si = species[i];
      const double* bs = beta + (size_t)K * si;
      compute_ui(s, nn, r, jn, si, species, w);
      compute_zi(s, w);
      compute_bi(s, w, si);
      if (s.quadratic_flag)
        quad_extend(s, w.b.data(), bx.data());
      else
        bx = w.b;
      double ei = 0.0;
      for (int q = 0; q < K; q++) ei += bs[q] * bx[q];
      Eth[tid] += ei;
      if (Ei) Ei[i] = ei;
      if (!F && !W6) continue;
      // forces need the linear coefficients only (quadratic: per-atom effective ones)
      if (s.quadratic_flag)
        quad_beta_eff(s, bs, w.b.data(), beff.data());
      else
        std::memcpy(beff.data(), bs, sizeof(double) * KL);
      const bool adj = mode == 1 && !s.chem_flag;  // the Y restatement covers one element
      if (adj) compute_yi(s, beff.data(), w);
      w.dur.assign((size_t)s.idxu_max * 3, 0.0);
      w.dui.assign((size_t)s.idxu_max * 3, 0.0);
      for (int64_t k = 0; k < nn; k++) {
        int32_t jj = jn[k];
        int32_t sj = species[jj];
        double rcut = (s.radii[si] + s.radii[sj]) * s.rcutfac;
        compute_duidrj(s, r + 3 * k, s.weight[sj], rcut, &w.ulr[(size_t)k * s.idxu_max],
                       &w.uli[(size_t)k * s.idxu_max], w.dur.data(), w.dui.data());
        double f[3] = {0.0, 0.0, 0.0};
        if (adj) {
          compute_deidrj(s, w, f);
        } else {
          compute_dbidrj(s, w, sj);
          for (int q = 0; q < KL; q++)
            for (int c = 0; c < 3; c++) f[c] += w.db[3 * q + c] * beff[q];
        }
        if (F)
          for (int c = 0; c < 3; c++) {
            Fth[tid][3 * i + c] += f[c];
            Fth[tid][3 * jj + c] -= f[c];
          }
        const double* xi = pos + 3 * i;
        const double* xj = pos + 3 * jj;
        double* wt = &Wth[6 * tid];
        wt[0] += f[0] * xi[0] - f[0] * xj[0];
        wt[1] += f[1] * xi[1] - f[1] * xj[1];
        wt[2] += f[2] * xi[2] - f[2] * xj[2];
        wt[3] += f[1] * xi[2] - f[1] * xj[2];
        wt[4] += f[0] * xi[2] - f[0] * xj[2];
        wt[5] += f[0] * xi[1] - f[0] * xj[1];
      }
    }
  }
  double Et = beta0;
  for (int t = 0; t < nt; t++) Et += Eth[t];
  if (E) *E = Et;
  if (F) {
    std::memset(F, 0, sizeof(double) * 3 * n);
    for (int t = 0; t < nt; t++)
      for (int64_t k = 0; k < 3 * n; k++) F[k] += Fth[t][k];
  }
  if (W6) {
    for (int c = 0; c < 6; c++) {
      W6[c] = 0.0;
      for (int t = 0; t < nt; t++) W6[c] += Wth[6 * t + c];
    }
  }
  return 0;
}

// Vector-Jacobian product of (E, F) with respect to beta: gbeta[s][k] =
// gE * sum_{i in s} B_i[k] + sum_k gF_k . dB_k[:, block s][k]; gbeta0 = gE.  The force part is
// sum over pairs (i, j) of (gF_i - gF_j) . dB_i/dr_ij in the block of s_i (the dB of
// compute_all_descriptors gathered per atom, snap.jl:276-277), summed per OpenMP thread.
int orc_snap_vjp_beta(void* h, int64_t n, const double* pos, const int32_t* species, const double* L, double gE,
                      const double* gF, double* gbeta, double* gbeta0) {
  Snap& s = *static_cast<Snap*>(h);
  int st = snap_check(s, n, pos, species, L);
  if (st) return st;
  PairList pl;
  snap_list(n, pos, L, species, s.nsp, s.radii.data(), s.rcutfac, s.literal_sqrt, pl);
  const int K = s.ncoef(), Kn = K * s.nsp;
#ifdef _OPENMP
  int nt = omp_get_max_threads();
#else
  int nt = 1;
#endif
  std::vector<std::vector<double>> gth(nt, std::vector<double>(Kn, 0.0));
#pragma omp parallel
  {
#ifdef _OPENMP
    int tid = omp_get_thread_num();
#else
    int tid = 0;
#endif
    AtomWork w;
    std::vector<double> bx(K), dbx(3 * (size_t)K);
    double* g = gth[tid].data();
#pragma omp for schedule(dynamic, 4)
    for (int64_t i = 0; i < n; i++) {
      int64_t nn = pl.off[i + 1] - pl.off[i];
      const double* r = &pl.r[3 * pl.off[i]];
      const int32_t* jn = &pl.j[pl.off[i]];
      int32_t si = species[i];
      compute_ui(s, nn, r, jn, si, species, w);
      compute_zi(s, w);
      compute_bi(s, w, si);
      if (s.quadratic_flag)
        quad_extend(s, w.b.data(), bx.data());
      else
        bx = w.b;
      double* gs = g + (size_t)K * si;
      for (int q = 0; q < K; q++) gs[q] += gE * bx[q];
      if (!gF) continue;
      w.dur.assign((size_t)s.idxu_max * 3, 0.0);
      w.dui.assign((size_t)s.idxu_max * 3, 0.0);
      for (int64_t k = 0; k < nn; k++) {
        int32_t jj = jn[k];
        int32_t sj = species[jj];
        double rcut = (s.radii[si] + s.radii[sj]) * s.rcutfac;
        compute_duidrj(s, r + 3 * k, s.weight[sj], rcut, &w.ulr[(size_t)k * s.idxu_max],
                       &w.uli[(size_t)k * s.idxu_max], w.dur.data(), w.dui.data());
        compute_dbidrj(s, w, sj);
        if (s.quadratic_flag)
          quad_extend_d(s, w.b.data(), w.db.data(), dbx.data());
        else
          dbx = w.db;
        const double gv[3] = {gF[3 * i] - gF[3 * jj], gF[3 * i + 1] - gF[3 * jj + 1], gF[3 * i + 2] - gF[3 * jj + 2]};
        for (int q = 0; q < K; q++) gs[q] += gv[0] * dbx[3 * q] + gv[1] * dbx[3 * q + 1] + gv[2] * dbx[3 * q + 2];
      }
    }
  }
  for (int c = 0; c < Kn; c++) {
    double t = 0.0;
    for (int q = 0; q < nt; q++) t += gth[q][c];
    gbeta[c] = t;
  }
  if (gbeta0) *gbeta0 = gE;
  return 0;
}

}  // extern "C"
