// ipg_pair.cu — fused multi-term empirical pair potentials.
//
// Replaces, for every term of a LinearCombinationPotential at once, the per-term
// neighbor build + pair loop of src/types/empirical_potential.jl:20-67 with one pass over
// the cell list at the largest cutoff, each term keeping its own cutoff (PeriodicEuclidean
// distance <= rcut_t, as the term's own neighbor list would) and species filter (both
// species in the term's set, empirical_potential.jl:26-43).
//
// Half-stencil tiles (k_pair_half).  Like the reference's half list (nnlist.jl:39-40, m > n),
// every unordered pair is evaluated once.  A work item is a (home cell A, offset k) pair,
// one warp each: k = 0 is A itself (pairs of slots s < s'), k = 1..13 the 13 neighbor cells
// of the forward half of the 27-cell stencil.  Lanes own the atoms of the target cell
// (positions in registers), the warp walks the home cell's atoms one row at a time (a
// broadcast load), the pairs within the largest cutoff are compacted into a per-warp hit
// buffer in (row, lane) order, and every 32 hits are evaluated by the whole warp.  The force
// of each hit goes to its two atoms' owner lanes by a broadcast loop in hit order, so every
// sum runs in a fixed order (no atomics).  A warp writes its row sums and column sums to its
// own slots of a partial-force buffer, [14 home offsets + 13 target offsets][slot][3], which
// k_pair_gather sums per atom in a fixed order.  Each pair's force term is the reference's:
// with lo < hi the atom ids, r = get_displacement(x_lo, x_hi) (nnlist.jl:18-21), f = g(R) r,
// F_lo += f, F_hi -= f; only the order of summation differs.
//
// The half stencil visits each pair of neighboring cells once only when every periodic axis
// has at least 3 cells; otherwise the full-stencil walk (ipg_pair.cuh) runs instead.
#include "ipg_pair.cuh"

namespace {

constexpr int PAIR_T = 128;
constexpr int PAIR_WARPS = PAIR_T / 32;

// The full-stencil walk, one warp per atom (the fallback for grids with fewer than 3 cells
// on a periodic axis).
__global__ void __launch_bounds__(PAIR_T) k_pair_eval(const __grid_constant__ PairTerms TT, int64_t n,
                                                      const ConfGrid* __restrict__ grid,
                                                      const int64_t* __restrict__ cell_start,
                                                      const int32_t* __restrict__ cell_atoms,
                                                      const double4* __restrict__ spos, double* __restrict__ F,
                                                      double* __restrict__ partial) {
  __shared__ PairHit hits[PAIR_WARPS][64];
  __shared__ double red[PAIR_WARPS][7];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t s = (int64_t)blockIdx.x * PAIR_WARPS + w;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};  // E, W[6]
  if (s < n) pair_walk_atom(TT, grid[0], cell_start, cell_atoms, spos, s, hits[w], lane, acc, F);  // warp-uniform
#pragma unroll
  for (int k = 0; k < 7; k++) {
    const double v = warp_sum(acc[k]);
    if (lane == 0) red[w][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < 7) {
    double v = 0.0;
    for (int q = 0; q < PAIR_WARPS; q++) v += red[q][threadIdx.x];
    partial[(int64_t)blockIdx.x * 7 + threadIdx.x] = v;
  }
}

// ---------------------------------------------------------------------------------
// Half-stencil tiles.
constexpr int HALF_OFFSETS = 14;  // self + 13 forward neighbors
constexpr int PBUF_SLOTS = 27;    // partial forces per atom: 14 as a home atom, 13 as a target

// Offset k of the half stencil: 0 = (0,0,0); 1..13 = the (dx,dy,dz) with dz > 0, or dz = 0
// and dy > 0, or dz = dy = 0 and dx > 0.
__device__ __forceinline__ void half_offset(int k, int& dx, int& dy, int& dz) {
  if (k == 0) {
    dx = dy = dz = 0;
  } else if (k == 1) {
    dx = 1, dy = 0, dz = 0;
  } else if (k <= 4) {
    dx = k - 3, dy = 1, dz = 0;  // k = 2, 3, 4 -> dx = -1, 0, 1
  } else {
    const int q = k - 5;  // 0..8
    dx = q % 3 - 1, dy = q / 3 - 1, dz = 1;
  }
}

// Cell coordinate c + d along an axis of nc cells: wrapped on a periodic axis (nc >= 3 there,
// so c + d stays a distinct cell), -1 when it leaves an open axis.
__device__ __forceinline__ int shift_axis(int c, int d, int nc, bool periodic) {
  int t = c + d;
  if (periodic) return t < 0 ? t + nc : (t >= nc ? t - nc : t);
  return (t < 0 || t >= nc) ? -1 : t;
}

struct HalfHit {
  double r0, r1, r2, dist;
  int at;  // row (bits 0-7) and lane (bits 8-15) within the tile
  int sp;  // species of the row atom (bits 0-7) and of the lane atom (bits 8-15)
};

// Per-warp staging of half_eval: a force per row and per column of the tile.
struct HalfStage {
  double row[32][3];
  double col[32][3];
};

// Evaluates the first nh hits (one per lane) and hands each hit's force to its row owner
// (fa += f) and its column owner (ft -= f).  Rows: the hits of a row are contiguous (they are
// appended in row order), so a segmented scan over the lanes (a fixed tree) leaves each row's
// total at its last hit, which stages it for the row's owner lane.  Columns: a row's hits have
// distinct columns, so the rows of the batch are handed over one after another (row order),
// each hit staging its force for its column's owner lane.  E and W accumulate lane-wise.
__device__ __forceinline__ void half_eval(const PairTerms& TT, const HalfHit* __restrict__ hb, int nh, int lane,
                                          HalfStage& st, double* acc, double* fa, double* ft) {
  constexpr unsigned FULL = 0xffffffffu;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  int row = 64 + lane, col = 0;  // idle lanes: rows that match no hit
  const bool act = lane < nh;
  if (act) {
    const HalfHit h = hb[lane];
    const double R = sqrt(h.r0 * h.r0 + h.r1 * h.r1 + h.r2 * h.r2);
    double V, g;
    pair_terms_sum(TT, R, h.dist, h.sp & 0xff, (h.sp >> 8) & 0xff, V, g);
    fx = g * h.r0;
    fy = g * h.r1;
    fz = g * h.r2;
    acc[0] += V;
    // empirical_potential.jl:63-64: r * f' -> [xx, yy, zz, zy, zx, yx]
    acc[1] += h.r0 * fx;
    acc[2] += h.r1 * fy;
    acc[3] += h.r2 * fz;
    acc[4] += h.r2 * fy;
    acc[5] += h.r2 * fx;
    acc[6] += h.r1 * fx;
    row = h.at & 0xff;
    col = (h.at >> 8) & 0xff;
  }
  // rows: segmented inclusive scan over the lanes
  double sx = fx, sy = fy, sz = fz;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double ox = __shfl_up_sync(FULL, sx, off), oy = __shfl_up_sync(FULL, sy, off),
                 oz = __shfl_up_sync(FULL, sz, off);
    const int orow = __shfl_up_sync(FULL, row, off);
    if (lane >= off && orow == row) {
      sx += ox;
      sy += oy;
      sz += oz;
    }
  }
  const int nrow = __shfl_down_sync(FULL, row, 1);
  const bool last = act && (lane == nh - 1 || nrow != row);
  if (last) {
    st.row[row][0] = sx;
    st.row[row][1] = sy;
    st.row[row][2] = sz;
  }
  const unsigned rows = __reduce_or_sync(FULL, last ? 1u << row : 0u);
  __syncwarp();
  if ((rows >> lane) & 1u) {
    fa[0] += st.row[lane][0];
    fa[1] += st.row[lane][1];
    fa[2] += st.row[lane][2];
  }
  // columns: one row of the batch at a time
  unsigned pend = __ballot_sync(FULL, act);
  while (pend) {
    const int r = __shfl_sync(FULL, row, __ffs(pend) - 1);
    const bool in = act && row == r;
    const unsigned seg = __ballot_sync(FULL, in);
    if (in) {
      st.col[col][0] = fx;
      st.col[col][1] = fy;
      st.col[col][2] = fz;
    }
    const unsigned cols = __reduce_or_sync(FULL, in ? 1u << col : 0u);
    __syncwarp();
    if ((cols >> lane) & 1u) {
      ft[0] -= st.col[lane][0];
      ft[1] -= st.col[lane][1];
      ft[2] -= st.col[lane][2];
    }
    __syncwarp();
    pend &= ~seg;
  }
}

__device__ __forceinline__ void pbuf_put(double* __restrict__ P, int64_t n, int slot_kind, int64_t s, const double* f,
                                         bool accumulate) {
  double* q = P + 3 * ((int64_t)slot_kind * n + s);
  if (accumulate) {
    q[0] += f[0];
    q[1] += f[1];
    q[2] += f[2];
  } else {
    q[0] = f[0];
    q[1] = f[1];
    q[2] = f[2];
  }
}

// MINB: resident blocks per SM the register allocation is bounded for (3: 168 registers, the
// default; 4: 128; 5: 96, with spills; 36.0 / 36.6 / 66 ms at 4.1 M atoms, five terms).
template <int MINB>
__global__ void __launch_bounds__(PAIR_T, MINB) k_pair_half(const __grid_constant__ PairTerms TT, int64_t n,
                                                         const ConfGrid* __restrict__ grid, int64_t ncells,
                                                         const int64_t* __restrict__ cell_start,
                                                         const int32_t* __restrict__ cell_atoms,
                                                         const double4* __restrict__ spos, double* __restrict__ P,
                                                         double* __restrict__ partial) {
  __shared__ HalfHit hits[PAIR_WARPS][64];
  __shared__ HalfStage stage[PAIR_WARPS];
  __shared__ double red[PAIR_WARPS][7];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};  // E, W[6] of every item this warp takes
  const double L0 = grid[0].L[0], L1 = grid[0].L[1], L2 = grid[0].L[2];
  // grid-stride over the items (a fixed assignment, so E and W sum in a fixed order); the
  // block's warps meet at a barrier only once, at the end
  const int64_t nitems = ncells * HALF_OFFSETS;
  const int64_t wstride = (int64_t)gridDim.x * PAIR_WARPS;
  for (int64_t item = (int64_t)blockIdx.x * PAIR_WARPS + w; item < nitems; item += wstride) {  // warp-uniform
    const ConfGrid& g = grid[0];
    // cells number below 2^31 (ipg_build_cells): 32-bit index arithmetic
    const int A = (int)(item / HALF_OFFSETS);
    const int k = (int)(item - (int64_t)A * HALF_OFFSETS);
    const int nxy = g.nc[0] * g.nc[1];
    const int cz = A / nxy, rem = A - cz * nxy;
    const int cy = rem / g.nc[0], cx = rem - cy * g.nc[0];
    int dx, dy, dz;
    half_offset(k, dx, dy, dz);
    const int tx = shift_axis(cx, dx, g.nc[0], !isinf(L0));
    const int ty = shift_axis(cy, dy, g.nc[1], !isinf(L1));
    const int tz = shift_axis(cz, dz, g.nc[2], !isinf(L2));
    if (tx < 0 || ty < 0 || tz < 0) continue;
    const int64_t T = ((int64_t)tz * g.nc[1] + ty) * g.nc[0] + tx;
    const int64_t a0 = cell_start[A], a1 = cell_start[A + 1], t0 = cell_start[T], t1 = cell_start[T + 1];
    const int home_kind = k, tgt_kind = k == 0 ? 0 : HALF_OFFSETS - 1 + k;
    // cells of at most 32 atoms are one tile and its sums are stored; larger cells take
    // several tiles, whose sums accumulate into zeroed slots, as do the row and column sums
    // of the home cell with itself (each slot is always written by the same lane, in tile
    // order)
    const bool multi = (a1 - a0 > 32) || (t1 - t0 > 32) || k == 0;
    if (multi) {
      const double z[3] = {0.0, 0.0, 0.0};
      for (int64_t s = a0 + lane; s < a1; s += 32) pbuf_put(P, n, home_kind, s, z, false);
      if (k != 0)
        for (int64_t s = t0 + lane; s < t1; s += 32) pbuf_put(P, n, tgt_kind, s, z, false);
      __syncwarp();
    }
    if (a0 == a1 && k != 0)  // no home atoms: the target atoms still get their (zero) slot
      for (int64_t s = t0 + lane; s < t1; s += 32) {
        const double z[3] = {0.0, 0.0, 0.0};
        pbuf_put(P, n, tgt_kind, s, z, false);
      }
    HalfHit* hb = hits[w];
    const unsigned lt = (1u << lane) - 1u;
    const double rmax = TT.rcut_max;
    for (int64_t rc = a0; rc < a1; rc += 32) {
      const int ra = (int)(a1 - rc < 32 ? a1 - rc : 32);
      double fa[3] = {0.0, 0.0, 0.0};  // row sums of row rc + lane
      for (int64_t cc = t0; cc < t1; cc += 32) {
        const int64_t ts = cc + lane;
        const bool tv = ts < t1;
        const double4 xt = tv ? spos[ts] : make_double4(0.0, 0.0, 0.0, 0.0);
        const int32_t it = tv ? cell_atoms[ts] : -1;
        double ft[3] = {0.0, 0.0, 0.0};  // column sums of lane atom ts
        int nh = 0;
        for (int q = 0; q <= ra; q++) {  // q == ra: evaluate what is left
          if (q < ra) {
            const int64_t as = rc + q;
            const double4 xa = spos[as];
            const int32_t ia = cell_atoms[as];
            bool ok = false;
            HalfHit h;
            if (tv && (k != 0 || ts > as)) {
              const double d2 = sumsq3_dev(pe_axis_dev(L0, xa.x, xt.x), pe_axis_dev(L1, xa.y, xt.y),
                                           pe_axis_dev(L2, xa.z, xt.z));
              if (d2 <= TT.rmax2_hi) {
                const double dist = sqrt(d2);
                if (dist <= rmax) {
                  ok = true;
                  h.dist = dist;
                  h.at = q | (lane << 8);
                  h.sp = (int)xa.w | ((int)xt.w << 8);
                  if (ia < it) {  // r = get_displacement(x_lo, x_hi) with the row atom lo
                    h.r0 = disp_axis_dev(L0, xa.x, xt.x);
                    h.r1 = disp_axis_dev(L1, xa.y, xt.y);
                    h.r2 = disp_axis_dev(L2, xa.z, xt.z);
                  } else {  // the lane atom is lo: r = -get_displacement(x_lane, x_row)
                    h.r0 = -disp_axis_dev(L0, xt.x, xa.x);
                    h.r1 = -disp_axis_dev(L1, xt.y, xa.y);
                    h.r2 = -disp_axis_dev(L2, xt.z, xa.z);
                  }
                }
              }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, ok);
            if (ok) hb[nh + __popc(bal & lt)] = h;
            nh += __popc(bal);
            __syncwarp();
          }
          // one call site of the term code: full batches, then the rest after the last row
          while (nh >= 32 || (q == ra && nh > 0)) {
            const int m = nh < 32 ? nh : 32;
            half_eval(TT, hb, m, lane, stage[w], acc, fa, ft);
            __syncwarp();
            if (lane < nh - m) hb[lane] = hb[m + lane];
            nh -= m;
            __syncwarp();
          }
        }
        if (tv) pbuf_put(P, n, tgt_kind, ts, ft, multi);
        __syncwarp();
      }
      if (lane < ra) pbuf_put(P, n, home_kind, rc + lane, fa, multi);
      __syncwarp();
    }
  }
#pragma unroll
  for (int q = 0; q < 7; q++) {
    const double v = warp_sum(acc[q]);
    if (lane == 0) red[w][q] = v;
  }
  __syncthreads();
  if (threadIdx.x < 7) {
    double v = 0.0;
    for (int q = 0; q < PAIR_WARPS; q++) v += red[q][threadIdx.x];
    partial[(int64_t)blockIdx.x * 7 + threadIdx.x] = v;
  }
}

// F of every atom: its 14 partial sums as a home atom (offsets k whose target cell exists)
// and its 13 as a target (offsets k whose home cell, its own cell - offset k, exists), in
// that fixed order.
__global__ void k_pair_gather(int64_t n, const ConfGrid* __restrict__ grid, const int32_t* __restrict__ cell_atoms,
                              const double4* __restrict__ spos, const double* __restrict__ P,
                              double* __restrict__ F) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const ConfGrid& g = grid[0];
  const double4 x = spos[s];
  int c[3];
  cell_coords(g, x.x, x.y, x.z, c);
  const bool per[3] = {!isinf(g.L[0]), !isinf(g.L[1]), !isinf(g.L[2])};
  double f0 = 0.0, f1 = 0.0, f2 = 0.0;
  for (int kind = 0; kind < PBUF_SLOTS; kind++) {
    const int k = kind < HALF_OFFSETS ? kind : kind - (HALF_OFFSETS - 1);
    const int sg = kind < HALF_OFFSETS ? 1 : -1;
    int d[3];
    half_offset(k, d[0], d[1], d[2]);
    bool ok = true;
    for (int a = 0; a < 3; a++) ok &= shift_axis(c[a], sg * d[a], g.nc[a], per[a]) >= 0;
    if (!ok) continue;
    const double* q = P + 3 * ((int64_t)kind * n + s);
    f0 += q[0];
    f1 += q[1];
    f2 += q[2];
  }
  const int64_t i = cell_atoms[s];
  F[3 * i] = f0;
  F[3 * i + 1] = f1;
  F[3 * i + 2] = f2;
}

// Deterministic final reduction of per-block partials (E and W6): one block, fixed order;
// component 0 goes to E, 1..6 to W6 (either may be null).
__global__ void k_reduce_partials(int64_t nblocks, int width, const double* __restrict__ partial,
                                  double* __restrict__ E, double* __restrict__ W6) {
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
    if (threadIdx.x == 0) {
      if (k == 0 && E) *E = sm[0];
      if (k > 0 && W6) W6[k - 1] = sm[0];
    }
    __syncthreads();
  }
}

int prepare_terms(ipg_ctx* ctx, const ipg_pair_term* terms, int nterms, PairTerms& pt) {
  char err[256];
  const int st = pair_prepare_terms(terms, nterms, pt, err, sizeof(err));
  return st == IPG_OK ? IPG_OK : ipg_fail(ctx, st, "%s", err);
}

int pair_eval_device(ipg_ctx* ctx, int64_t n, const double* d_pos, const int32_t* d_species, const double L[3],
                     const ipg_pair_term* terms, int32_t nterms, double* d_E, double* d_F, double* d_W6,
                     uint32_t flags, std::vector<ConfGrid>* grid_out = nullptr) {
  PairTerms pt;
  IPG_RET(prepare_terms(ctx, terms, nterms, pt));
  IPG_RET(ipg_status_reset(ctx));
  int64_t aoff[2] = {0, n};
  CellList cl;
  IPG_RET(ipg_build_cells(ctx, "pair_", n, d_pos, d_species, 64, 1, aoff, L, pt.rcut_max, cl));
  if (grid_out) *grid_out = cl.h_grid;
  const ConfGrid& g = cl.h_grid[0];
  bool half = n > 0 && !ctx->pair_full_stencil;
  for (int a = 0; a < 3; a++) half &= std::isinf(g.L[a]) || g.nc[a] >= 3;
  double* partial;
  int64_t nb;
  IPG_RET(ipg_timing_mark(ctx, "pair_eval", true));
  if (half) {
    const int64_t items = cl.ncells * HALF_OFFSETS;
    // grid-stride: a fixed grid of a few waves of resident blocks (the kernel's register bound
    // allows pair_minb blocks of four warps per SM)
    nb = std::max<int64_t>(1, std::min<int64_t>((items + PAIR_WARPS - 1) / PAIR_WARPS,
                                                (int64_t)ctx->num_sms * ctx->pair_minb * 4));
    double* P;
    IPG_RET(scratch(ctx, "pair_partial", (size_t)nb * 7, &partial));
    IPG_RET(scratch(ctx, "pair_pbuf", (size_t)PBUF_SLOTS * 3 * n, &P));
    if (ctx->pair_minb == 4)
      IPG_LAUNCH(ctx, k_pair_half<4>, (unsigned)nb, PAIR_T, 0, pt, n, cl.d_grid, cl.ncells, cl.d_cell_start,
                 cl.d_cell_atoms, cl.d_spos, P, partial);
    else if (ctx->pair_minb == 5)
      IPG_LAUNCH(ctx, k_pair_half<5>, (unsigned)nb, PAIR_T, 0, pt, n, cl.d_grid, cl.ncells, cl.d_cell_start,
                 cl.d_cell_atoms, cl.d_spos, P, partial);
    else
      IPG_LAUNCH(ctx, k_pair_half<3>, (unsigned)nb, PAIR_T, 0, pt, n, cl.d_grid, cl.ncells, cl.d_cell_start,
                 cl.d_cell_atoms, cl.d_spos, P, partial);
    if ((flags & IPG_WANT_F) && d_F)
      IPG_LAUNCH(ctx, k_pair_gather, (unsigned)((n + 255) / 256), 256, 0, n, cl.d_grid, cl.d_cell_atoms, cl.d_spos,
                 P, d_F);
  } else {
    nb = std::max<int64_t>(1, (n + PAIR_WARPS - 1) / PAIR_WARPS);
    IPG_RET(scratch(ctx, "pair_partial", (size_t)nb * 7, &partial));
    IPG_LAUNCH(ctx, k_pair_eval, (unsigned)nb, PAIR_T, 0, pt, n, cl.d_grid, cl.d_cell_start, cl.d_cell_atoms,
               cl.d_spos, (flags & IPG_WANT_F) ? d_F : nullptr, partial);
  }
  IPG_RET(ipg_timing_mark(ctx, "pair_eval", false));
  IPG_LAUNCH(ctx, k_reduce_partials, 1, 256, 0, nb, 7, partial, (flags & IPG_WANT_E) ? d_E : nullptr,
             (flags & IPG_WANT_W) ? d_W6 : nullptr);
  return IPG_OK;
}

// ---- CUDA graphs of the device evaluation (IPG_PAIR_GRAPH) --------------------------------
ipg_ctx::PairGraph* pair_graph_find(ipg_ctx* ctx, int64_t n, const double* d_pos, const int32_t* d_species,
                                    const double L[3], const ipg_pair_term* terms, int32_t nterms,
                                    const double* d_E, const double* d_F, const double* d_W6, uint32_t flags) {
  const size_t tb = sizeof(ipg_pair_term) * (size_t)nterms;
  for (auto& g : ctx->pair_graphs)
    if (g.n == n && g.L[0] == L[0] && g.L[1] == L[1] && g.L[2] == L[2] && g.pos == d_pos && g.sp == d_species &&
        g.E == d_E && g.F == d_F && g.W6 == d_W6 && g.flags == flags && g.terms.size() == tb &&
        memcmp(g.terms.data(), terms, tb) == 0 && g.full_stencil == (int)ctx->pair_full_stencil &&
        g.minb == ctx->pair_minb)
      return &g;
  return nullptr;
}

// Uploads the cell grid the graph reads and launches it; IPG_ERR_NOT_CAPTURED when there is
// no usable graph (none for this key, or a scratch buffer moved since the capture).
int pair_graph_replay(ipg_ctx* ctx, int64_t n, const double* d_pos, const int32_t* d_species, const double L[3],
                      const ipg_pair_term* terms, int32_t nterms, double* d_E, double* d_F, double* d_W6,
                      uint32_t flags) {
  ipg_ctx::PairGraph* g = pair_graph_find(ctx, n, d_pos, d_species, L, terms, nterms, d_E, d_F, d_W6, flags);
  if (!g) return IPG_ERR_NOT_CAPTURED;
  ConfGrid* d_grid = nullptr;
  if (g->gen == ctx->scratch_gen) IPG_RET(scratch(ctx, "pair_grid", 1, &d_grid));
  if (g->gen != ctx->scratch_gen) {
    cudaGraphExecDestroy(g->exec);
    ctx->pair_graphs.erase(ctx->pair_graphs.begin() + (g - ctx->pair_graphs.data()));
    return IPG_ERR_NOT_CAPTURED;
  }
  CUDA_RET(ctx, cudaMemcpyAsync(d_grid, g->grid.data(), g->grid.size(), cudaMemcpyHostToDevice, ctx->stream));
  IPG_RET(ipg_status_reset(ctx));
  CUDA_RET(ctx, cudaGraphLaunch(g->exec, ctx->stream));
  ctx->pair_graph_replays++;
  return ipg_status_check(ctx, "ipg_pair_eval_dev (graph)");
}

// Captures the evaluation just run eagerly with the same inputs (every scratch buffer already
// has its size).  A failure only means that later calls run eagerly.
void pair_graph_capture(ipg_ctx* ctx, int64_t n, const double* d_pos, const int32_t* d_species, const double L[3],
                        const ipg_pair_term* terms, int32_t nterms, double* d_E, double* d_F, double* d_W6,
                        uint32_t flags) {
  if (ctx->pair_graphs.size() >= 8) {
    cudaGraphExecDestroy(ctx->pair_graphs.front().exec);
    ctx->pair_graphs.erase(ctx->pair_graphs.begin());
  }
  ipg_ctx::PairGraph g;
  g.n = n;
  for (int a = 0; a < 3; a++) g.L[a] = L[a];
  g.pos = d_pos;
  g.sp = d_species;
  g.E = d_E;
  g.F = d_F;
  g.W6 = d_W6;
  g.flags = flags;
  g.terms.assign(reinterpret_cast<const char*>(terms), reinterpret_cast<const char*>(terms) + sizeof(ipg_pair_term) * nterms);
  g.full_stencil = ctx->pair_full_stencil;
  g.minb = ctx->pair_minb;
  const uint64_t gen0 = ctx->scratch_gen;
  std::vector<ConfGrid> grid;
  const bool timing = ctx->timing;
  ctx->timing = false;
  ctx->capturing = true;
  cudaGraph_t graph = nullptr;
  int st = IPG_OK;
  if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
    st = IPG_ERR_CUDA;
  } else {
    st = pair_eval_device(ctx, n, d_pos, d_species, L, terms, nterms, d_E, d_F, d_W6, flags, &grid);
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    if (st == IPG_OK && e != cudaSuccess) st = IPG_ERR_CUDA;
  }
  ctx->capturing = false;
  ctx->timing = timing;
  if (st == IPG_OK && graph && ctx->scratch_gen == gen0 && grid.size() == 1 &&
      cudaGraphInstantiate(&g.exec, graph, 0) == cudaSuccess) {
    g.grid.assign(reinterpret_cast<const char*>(grid.data()), reinterpret_cast<const char*>(grid.data() + 1));
    g.gen = ctx->scratch_gen;
    ctx->pair_graphs.push_back(std::move(g));
  }
  if (graph) cudaGraphDestroy(graph);
  cudaGetLastError();  // a failed capture leaves no sticky error behind
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
    IPG_RET(ipg_copy_h2d(ctx, d_pos, pos, sizeof(double) * 3 * n));
    IPG_RET(ipg_copy_h2d(ctx, d_sp, species, sizeof(int32_t) * n));
  }
  // d_out layout: [E, W6 (6), pad, F (3n)]
  IPG_RET(pair_eval_device(ctx, n, d_pos, d_sp, L, terms, nterms, d_out, d_out + 8, d_out + 1,
                           flags | IPG_WANT_E | IPG_WANT_W));
  std::vector<double> head(8);
  CUDA_RET(ctx, cudaMemcpyAsync(head.data(), d_out, sizeof(double) * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if ((flags & IPG_WANT_F) && n) IPG_RET(ipg_copy_d2h(ctx, F, d_out + 8, sizeof(double) * 3 * n));
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
  const bool want_graph = (flags & IPG_PAIR_GRAPH) && n > 0 && !std::isinf(L[0]) && !std::isinf(L[1]) &&
                          !std::isinf(L[2]);
  flags &= IPG_WANT_E | IPG_WANT_F | IPG_WANT_W;
  if (want_graph) {
    const int st = pair_graph_replay(ctx, n, d_pos, d_species, L, terms, nterms, d_E, d_F, d_W6, flags);
    if (st != IPG_ERR_NOT_CAPTURED) return st;
  }
  IPG_RET(pair_eval_device(ctx, n, d_pos, d_species, L, terms, nterms, d_E, d_F, d_W6, flags));
  IPG_RET(ipg_status_check(ctx, "ipg_pair_eval_dev"));
  if (want_graph) pair_graph_capture(ctx, n, d_pos, d_species, L, terms, nterms, d_E, d_F, d_W6, flags);
  return IPG_OK;
}

}  // extern "C"
