// ipg_snap.cuh — SNAP tables and device-side descriptor of a SNAP basis.
#pragma once

#include "ipg_internal.cuh"

// One Z entry (one (j1, j2, j, ma, mb) of the idxz list, prebuilt_arrays.jl:183-216),
// with the start offsets of its CG double sum precomputed.
struct ZDev {
  int8_t j1, j2, j, na, nb, pad0, pad1, pad2;  // twojmax <= 12 bounds every index
  int8_t ma1min, ma2max, mb1min, mb2max;       // row/column starts of the two U factors
  int32_t u1base;  // idxu_block[j1] + (j1+1)*mb1min + ma1min
  int32_t u2base;  // idxu_block[j2] + (j2+1)*mb2max + ma2max
  int32_t icga0;   // ma1min*(j2+1) + ma2max
  int32_t icgb0;   // mb1min*(j2+1) + mb2max
  int32_t cgoff;   // idxcg_block[j1][j2][j]
};
static_assert(sizeof(ZDev) == 32, "ZDev is read as two 16-byte words");

// One bispectrum component (j1, j2, j) and the three half-plane sums of its
// derivative (compute_b.jl:207-400): level l[t], first Z index z0[t], factor fac[t].
struct DBDev {
  int32_t l[3];
  int32_t z0[3];
  double fac[3];
};

constexpr int SNAP_MAX_J = 12;
constexpr int YS_WARPS = 8;     // warps of the atoms-in-lanes Y kernels
constexpr int YS_ATOMS = 32;    // atoms per block of those kernels (one per lane)
constexpr int YR_MAX_J = 8;     // largest twojmax of the row-blocked Y kernel
constexpr int yr_rows(int J) { return J < 0 ? 0 : yr_rows(J - 1) + J / 2 + 1; }  // target rows (j, mb <= j/2)

// Row-blocked Y kernel: a target row (j, mb) of the half plane of Y and the (j1, j2)
// triples whose Z entries feed it.
struct YRowDev {
  int8_t j, mb, mid, pad;  // mid: middle row of an even level (weights vanish beyond ma = mb)
  int32_t h0;              // half-plane index of (j, mb, ma = 0)
  int32_t t0, t1;          // its triples: yitems[t0 .. t1)
};
struct YItemDev {
  int8_t j1, j2, d, nb, mb1min, mb2max, pad0, pad1;  // d = (j1 + j2 - j) / 2
  int32_t ca;   // offset in yca of the triple's CG factors, [m0/2][ma][2] (zero where out of range)
  int32_t cg;   // idxcg_block[j1][j2][j]: the row factors cg[mb1 (j2+1) + mb2]
  int32_t jjz;  // first Z entry of the triple (its Y coefficient)
  int32_t trip; // index of the triple (its coefficient slot in the kernel's shared table)
};
static_assert(sizeof(YItemDev) == 24, "YItemDev layout");

// The row-blocked Y kernel's warp-uniform tables, passed by value as a kernel parameter
// (constant bank: uniform reads through the constant cache, private to each launch).
constexpr int YC_ROWS = 28, YC_ITEMS = 400, YC_RP = 1536;
struct YConst {
  YRowDev rows[YC_ROWS];    // target rows, longest first
  YItemDev items[YC_ITEMS]; // their triples (field cg: offset of the first row factor in cb)
  double cb[YC_RP];         // cg[mb1][mb2] of every row pair of every item
  int nrows, nitems, nrp, pad;
};

struct SnapDev {
  int J, nsp, K, idxu_max, idxz_max, u_half, ext_max, idxcg_max;
  int switch_flag, bzero_flag, bnorm_flag, n_yrows;
  int n_ytrip, n_yca;  // row-blocked Y kernel: triples, doubles in yca
  double rcutfac, rmin0, rfac0, wself;
  double radii[IPG_MAX_SNAP_SPECIES], weight[IPG_MAX_SNAP_SPECIES];
  int idxu_block[SNAP_MAX_J + 2];
  int half_block[SNAP_MAX_J + 2];
  double bzero[SNAP_MAX_J + 1];
  const double* rootpq;  // [(J+2)*(J+2)]
  const double* cglist;  // [idxcg_max]
  const ZDev* idxz;      // [idxz_max]
  const DBDev* db;       // [K]
  const int32_t* y_off;  // [u_half+1]  CSR: Z entries feeding each half-plane Y entry
  const int32_t* y_jjz;  // [idxz_max]
  const double* ycoef;   // [nsp][idxz_max] multiplicity * factor * beta (set per beta)
  const double* beta;    // [nsp][K]
  const int32_t* zperm;  // [idxz_max] Z entries ordered by loop shape (nb, na)
  // Y schedule of the atoms-in-lanes kernel: warp w owns half-plane entries
  // ysched_h[ysched_off[w] .. ysched_off[w+1]) (cost-balanced), ysched_w their weights
  const int32_t* ysched_off;  // [YS_WARPS+1]
  const int32_t* ysched_h;
  const double* ysched_w;
  const int32_t* u_of_h;      // [u_half] index of half-plane entry h in the full Utot
  const int32_t* h_info;      // [u_half] m | j << 8 | (m within the row's weighted entries) << 16, m = column ma
  const double2* h_sgen;      // [u_half] the generator factors (s_m, s_{m-1}), s_m = sqrt((m+1)(j-m)), 0 off the row
  // row-blocked Y kernel (twojmax <= YR_MAX_J): n_yrows target rows, longest first
  const YRowDev* yrows;
  const YItemDev* yitems;
  const double* yca;
  const int32_t* ytrip_jjz;  // [n_ytrip] first Z entry of each triple
  // explicit multi-element SNAP (chem_flag) and quadratic SNAP: K is then the number of
  // components per species block, klin of them linear (idxb_max per element triple), the rest
  // the products B_k B_l (k <= l) of quadratic_flag
  int chem, nelem, wselfall, literal_chem_z, quadratic, klin;
  const double* beta0;  // [1] energy offset of LBasisPotential (device, like ebias)
  const double* ebias;  // [nsp] -beta[s] . bzero (energy shift of bzero_flag), device memory so that
                        // a captured graph sees the beta of each replay
};

struct SnapHost {
  int J = 0, idxu_max = 0, idxz_max = 0, idxb_max = 0, idxcg_max = 0, u_half = 0, ext_max = 0;
  std::vector<int> idxu_block, half_block, idxcg_block, idxz_block, idxb_block;
  std::vector<int> idxb;  // 3 per component
  std::vector<ZDev> idxz;
  std::vector<int> zjju_half;  // half-plane index of each Z entry
  std::vector<DBDev> db;
  std::vector<double> cglist, rootpq, bzero;
  std::vector<int32_t> y_off, y_jjz;
  std::vector<int32_t> y_jjb;     // component whose beta scales each Z entry in Y
  std::vector<double> y_mult;     // multiplicity * (j1+1)/(j+1) factor of each Z entry
  std::vector<int32_t> zperm;     // Z entries sorted by (nb, na): equal trip counts per warp
  std::vector<int32_t> ysched_off, ysched_h, u_of_h, h_info;
  std::vector<double> h_sgen;  // 2 per half-plane entry
  std::vector<double> ysched_w;
  std::vector<YRowDev> yrows;
  std::vector<YItemDev> yitems;
  std::vector<double> yca;
  std::vector<int32_t> ytrip_jjz;
  bool yconst_ok = false;  // the tables fit YConst
  YConst yconst;
};

int snap_build_tables(const ipg_snap_params& p, SnapHost& h);
