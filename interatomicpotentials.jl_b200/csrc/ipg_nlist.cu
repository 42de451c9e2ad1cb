// ipg_nlist.cu — cell-list neighbor build (replaces the BallTree + PeriodicEuclidean
// search of src/nnlist.jl:23-46 and src/BasisSystems/SNAP/utilities/utl.jl:38-101).
//
// Pipeline (all on the context's stream):
//   k_extent       per-configuration min/max of open axes (only when an axis is open)
//   k_cell_count   cell id per atom + histogram
//   scan           cell_start
//   k_cell_fill    scatter atom ids into their cells
//   k_cell_sort    sort each cell ascending (deterministic slot order), slot_of, spos
// and, for a materialised list:
//   k_pair_count / scan / k_pair_emit / k_pair_sort, optionally the transpose.
// Membership is decided per candidate with the reference's own arithmetic
// (PeriodicEuclidean distance, get_displacement), so any cell edge >= the search radius
// proposes every pair exactly once.
#include <algorithm>

#include "ipg_internal.cuh"

namespace {

__global__ void k_extent(const double* __restrict__ pos, const ConfGrid* __restrict__ grid, double* __restrict__ ext) {
  // one block per configuration; ext[c*6 + a] = min, ext[c*6 + 3 + a] = max
  const ConfGrid g = grid[blockIdx.x];
  __shared__ double smin[3][32], smax[3][32];
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t i = threadIdx.x; i < g.natoms; i += blockDim.x) {
    const double* p = pos + 3 * (g.atom_off + i);
#pragma unroll
    for (int a = 0; a < 3; a++) {
      mn[a] = fmin(mn[a], p[a]);
      mx[a] = fmax(mx[a], p[a]);
    }
  }
#pragma unroll
  for (int a = 0; a < 3; a++)
    for (int o = 16; o > 0; o >>= 1) {
      mn[a] = fmin(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
      mx[a] = fmax(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
    }
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0)
    for (int a = 0; a < 3; a++) {
      smin[a][w] = mn[a];
      smax[a][w] = mx[a];
    }
  __syncthreads();
  if (threadIdx.x < 3) {
    int a = threadIdx.x;
    double m = INFINITY, M = -INFINITY;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) {
      m = fmin(m, smin[a][q]);
      M = fmax(M, smax[a][q]);
    }
    ext[blockIdx.x * 6 + a] = m;
    ext[blockIdx.x * 6 + 3 + a] = M;
  }
}

__global__ void k_cell_count(int64_t n, const double* __restrict__ pos, const int32_t* __restrict__ species, int nsp,
                             const ConfGrid* __restrict__ grid, int nconf, int32_t* __restrict__ conf,
                             int32_t* __restrict__ cell_of, int64_t* __restrict__ count, int* status) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // configuration by binary search over atom offsets
  int lo = 0, hi = nconf - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (grid[mid].atom_off <= i) lo = mid;
    else hi = mid - 1;
  }
  const ConfGrid& g = grid[lo];
  double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
  if (!isfinite(x) || !isfinite(y) || !isfinite(z)) {
    dev_raise(status, IPG_ERR_NONFINITE);
    x = y = z = 0.0;
  }
  if (species && (species[i] < 0 || species[i] >= nsp)) dev_raise(status, IPG_ERR_SPECIES);
  int c[3];
  cell_coords(g, x, y, z, c);
  int64_t cell = g.cell_off + ((int64_t)c[2] * g.nc[1] + c[1]) * g.nc[0] + c[0];
  conf[i] = lo;
  cell_of[i] = (int32_t)cell;
  atomicAdd((unsigned long long*)&count[cell], 1ull);
}

__global__ void k_cell_fill(int64_t n, const int32_t* __restrict__ cell_of, const int64_t* __restrict__ cell_start,
                            int64_t* __restrict__ fill, int32_t* __restrict__ cell_atoms) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t c = cell_of[i];
  unsigned long long q = atomicAdd((unsigned long long*)&fill[c], 1ull);
  cell_atoms[cell_start[c] + (int64_t)q] = (int32_t)i;
}

__global__ void k_cell_sort(int64_t ncells, const int64_t* __restrict__ cell_start, int32_t* __restrict__ cell_atoms) {
  int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  int64_t s = cell_start[c], e = cell_start[c + 1];
  for (int64_t a = s + 1; a < e; a++) {
    int32_t v = cell_atoms[a];
    int64_t b = a - 1;
    while (b >= s && cell_atoms[b] > v) {
      cell_atoms[b + 1] = cell_atoms[b];
      b--;
    }
    cell_atoms[b + 1] = v;
  }
}

__global__ void k_cell_gather(int64_t n, const int32_t* __restrict__ cell_atoms, const double* __restrict__ pos,
                              const int32_t* __restrict__ species, int nsp, int32_t* __restrict__ slot_of,
                              double4* __restrict__ spos) {
  int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  int32_t i = cell_atoms[s];
  slot_of[i] = (int32_t)s;
  int sp = species ? species[i] : 0;
  sp = sp < 0 ? 0 : (sp > nsp - 1 ? nsp - 1 : sp);  // bad ids were reported by k_cell_count
  spos[s] = make_double4(pos[3 * (int64_t)i], pos[3 * (int64_t)i + 1], pos[3 * (int64_t)i + 2], (double)sp);
}

// ---------------------------------------------------------------------------------
// Pair tests.  HALF: nnlist.jl:39-44.  FULL: utl.jl:81-93.
struct PairTest {
  int mode;          // IPG_NLIST_HALF / IPG_NLIST_FULL
  int literal;       // utl.jl:81 literal search radius
  int nsp;
  double rcut;       // HALF: cutoff; FULL: candidate radius (cutmax or sqrt(cutmax))
  double rcut2_lo, rcut2_hi;  // rcut^2 (1 -/+ 1e-12)
  double cutsq[64];  // FULL: [nsp][nsp], nsp <= 8
};

// Returns true when (i, j) belongs to the list; r receives the stored displacement.
__device__ __forceinline__ bool pair_ok(const PairTest& t, const double* L, int32_t i, double4 xi, int32_t j,
                                        double4 xj, double* r) {
  if (t.mode == IPG_NLIST_HALF) {
    if (j <= i) return false;
  } else if (j == i) {
    return false;
  }
  double s0 = pe_axis_dev(L[0], xi.x, xj.x);
  double s1 = pe_axis_dev(L[1], xi.y, xj.y);
  double s2 = pe_axis_dev(L[2], xi.z, xj.z);
  // sqrt(d2) <= rcut decided exactly; the squared bounds (1e-12 relative margin, far
  // above the rounding of sqrt and of rcut^2) settle all but the boundary cases
  const double d2 = sumsq3_dev(s0, s1, s2);
  if (d2 > t.rcut2_hi) return false;
  if (d2 >= t.rcut2_lo && sqrt(d2) > t.rcut) return false;
  r[0] = disp_axis_dev(L[0], xi.x, xj.x);
  r[1] = disp_axis_dev(L[1], xi.y, xj.y);
  r[2] = disp_axis_dev(L[2], xi.z, xj.z);
  if (t.mode == IPG_NLIST_HALF) return true;
  r[0] = -r[0];
  r[1] = -r[1];
  r[2] = -r[2];
  double rsq = sumsq3_dev(r[0], r[1], r[2]);
  return rsq <= t.cutsq[(int)xi.w * t.nsp + (int)xj.w];
}

// One warp per atom (cell-sorted order): lanes take consecutive candidates of each
// stencil range (coalesced), ballots count the members, and the emit pass writes them
// in candidate order (ballot prefix), so the list is deterministic.
template <bool EMIT>
__global__ void __launch_bounds__(128) k_pair_walk(int64_t n, PairTest t, const ConfGrid* __restrict__ grid,
                                                   const int32_t* __restrict__ conf,
                                                   const int64_t* __restrict__ cell_start,
                                                   const int32_t* __restrict__ cell_atoms,
                                                   const double4* __restrict__ spos, int64_t* __restrict__ cnt,
                                                   const int64_t* __restrict__ off, int32_t* __restrict__ outj,
                                                   double* __restrict__ outr) {
  const int lane = threadIdx.x & 31;
  const int64_t s = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (s >= n) return;  // warp-uniform
  const int32_t i = cell_atoms[s];
  const double4 xi = spos[s];
  const ConfGrid g = grid[conf[i]];
  int c[3];
  cell_coords(g, xi.x, xi.y, xi.z, c);
  StencilRanges R;
  stencil_ranges(g, c, cell_start, R);
  int64_t k = 0;
  const int64_t base = EMIT ? off[i] : 0;
  const int64_t end = EMIT ? off[i + 1] : 0;
  const unsigned lt = (1u << lane) - 1u;
  for (int r = 0; r < R.n; r++)
    for (int64_t q0 = R.beg[r]; q0 < R.end[r]; q0 += 32) {
      const int64_t q = q0 + lane;
      double rr[3];
      bool ok = false;
      if (q < R.end[r]) ok = pair_ok(t, g.L, i, xi, cell_atoms[q], spos[q], rr);
      const unsigned bal = __ballot_sync(0xffffffffu, ok);
      if (EMIT && ok) {
        const int64_t o = base + k + __popc(bal & lt);
        if (o < end) {  // a list cut at the capacity (capacity mode) drops its tail
          outj[o] = cell_atoms[q];
          outr[3 * o] = rr[0];
          outr[3 * o + 1] = rr[1];
          outr[3 * o + 2] = rr[2];
        }
      }
      k += __popc(bal);
    }
  if (!EMIT && lane == 0) cnt[i] = k;
}

// Verlet-skin reuse: the pairs of a list built with enlarged cutoffs that satisfy the true
// test (pair_ok, the same arithmetic as a fresh build) at the current positions.  One warp
// per atom, lanes over its cached candidates, emission in the cached order.
template <bool EMIT>
__global__ void __launch_bounds__(128) k_filter_walk(int64_t n, PairTest t, const ConfGrid* __restrict__ grid,
                                                     const int32_t* __restrict__ conf,
                                                     const int64_t* __restrict__ coff,
                                                     const int32_t* __restrict__ cj, const double* __restrict__ pos,
                                                     const int32_t* __restrict__ species, int nsp,
                                                     int64_t* __restrict__ cnt, const int64_t* __restrict__ off,
                                                     int32_t* __restrict__ outj, double* __restrict__ outr,
                                                     int* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= n) return;  // warp-uniform
  // ids are clamped so every table read stays in bounds; an id out of range is an error
  if (!EMIT && lane == 0 && species && (species[i] < 0 || species[i] >= nsp)) dev_raise(status, IPG_ERR_SPECIES);
  const int si = species ? (species[i] < 0 ? 0 : (species[i] >= nsp ? nsp - 1 : species[i])) : 0;
  const double4 xi = make_double4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], (double)si);
  const double* L = grid[conf[i]].L;
  int64_t k = 0;
  const int64_t base = EMIT ? off[i] : 0;
  const unsigned lt = (1u << lane) - 1u;
  for (int64_t q0 = coff[i]; q0 < coff[i + 1]; q0 += 32) {
    const int64_t q = q0 + lane;
    double rr[3];
    bool ok = false;
    int32_t j = 0;
    if (q < coff[i + 1]) {
      j = cj[q];
      const int sj = species ? (species[j] < 0 ? 0 : (species[j] >= nsp ? nsp - 1 : species[j])) : 0;
      ok = pair_ok(t, L, (int32_t)i, xi, j, make_double4(pos[3 * j], pos[3 * j + 1], pos[3 * j + 2], (double)sj), rr);
    }
    const unsigned bal = __ballot_sync(0xffffffffu, ok);
    if (EMIT && ok) {
      const int64_t o = base + k + __popc(bal & lt);
      outj[o] = j;
      outr[3 * o] = rr[0];
      outr[3 * o + 1] = rr[1];
      outr[3 * o + 2] = rr[2];
    }
    k += __popc(bal);
  }
  if (!EMIT && lane == 0) cnt[i] = k;
}

// Largest squared minimum-image displacement since the reference positions, as the bit
// pattern of a non-negative double (ordered like the integers).  A non-finite position, or a
// species id that differs from the one at the build, counts as an infinite move, so the
// caller rebuilds the list (and the fresh build reports the bad input).
__global__ void k_max_disp2(int64_t n, const ConfGrid* __restrict__ grid, const int32_t* __restrict__ conf,
                            const double* __restrict__ pos, const double* __restrict__ ref,
                            const int32_t* __restrict__ species, const int32_t* __restrict__ ref_species,
                            unsigned long long* __restrict__ out) {
  __shared__ unsigned long long sm[256];
  double m = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double* L = grid[conf[i]].L;
    double d2 = 0.0;
    for (int a = 0; a < 3; a++) {
      const double s = pe_axis_dev(L[a], pos[3 * i + a], ref[3 * i + a]);
      d2 += s * s;
    }
    if (!(d2 <= 1.7976931348623157e308)) d2 = INFINITY;  // NaN or Inf: never reuse
    if (species && ref_species && species[i] != ref_species[i]) d2 = INFINITY;
    m = fmax(m, d2);
  }
  sm[threadIdx.x] = (unsigned long long)__double_as_longlong(m);
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sm[threadIdx.x] = sm[threadIdx.x] > sm[threadIdx.x + o] ? sm[threadIdx.x] : sm[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicMax(out, sm[0]);
}

// Capacity mode: a total above cap is an error (status), and every offset is cut at cap
// so that all later kernels stay inside the buffers.
// (Offsets are non-decreasing, so cutting each one at cap on its own is the same as
// cutting the lists; no thread reads another's offset.)
__global__ void k_clamp_offsets(int64_t n, int64_t* __restrict__ off, int64_t cap, int* __restrict__ status) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i > n) return;
  if (off[i] > cap) {
    if (i == n) atomicExch(status, IPG_ERR_CAPACITY);
    off[i] = cap;
  }
}

// The same walk with one warp per cell: every atom of a cell has the same stencil, so each
// chunk of 32 candidates is loaded once and tested against every atom of a group of up to 32
// atoms of the cell, in two phases.  Phase 1 applies only the first test of pair_ok (the
// periodic distance against the candidate radius, with the same arithmetic, so the same
// decision; a separation of a box length or more is left to the full test), WALK_ILP atoms at
// a time so that their independent FP64 chains overlap, and queues the (atom, candidate) pairs
// that pass in (atom, lane) order in a per-warp ring.  Phase 2 runs the full pair_ok on 32
// queued pairs at a time, one per lane, and emits the members after each atom's running count
// (shared memory).  One test in eight passes: with the member path inside the chunk loop, the
// few members of a chunk made every lane run it.  Each atom's hits come out in candidate order,
// as from k_pair_walk.
constexpr int WALKC_WARPS = 4;
constexpr int WALK_ILP = 4;    // atoms per phase-1 step
constexpr int WALK_RING = 256;  // queue entries per warp (a step adds at most 32 * WALK_ILP to fewer than 32)
struct WalkAtom {
  double4 x;
  int64_t base, end;
  int32_t i, cnt;  // atom id, hits so far
};
struct WalkQ {
  int32_t slot, ii;  // candidate slot, group atom
};

// The first test of pair_ok: false only when pair_ok is false.  Branch-free: every term is
// formed, and the flags are combined bitwise.
__device__ __forceinline__ bool walk_prefilter(const PairTest& t, const double* L, int32_t i, double4 xi, int32_t j,
                                               double4 xj) {
  const bool other = t.mode == IPG_NLIST_HALF ? j > i : j != i;
  // pe_axis_dev for |a - b| < L (an open axis has L = inf, where min(s1, inf) = s1)
  const double s0 = fabs(__dsub_rn(xi.x, xj.x)), s1 = fabs(__dsub_rn(xi.y, xj.y)), s2 = fabs(__dsub_rn(xi.z, xj.z));
  const bool far = !(s0 < L[0]) | !(s1 < L[1]) | !(s2 < L[2]);  // fmod case or NaN: full test
  const double m0 = fmin(s0, __dsub_rn(L[0], s0)), m1 = fmin(s1, __dsub_rn(L[1], s1)),
               m2 = fmin(s2, __dsub_rn(L[2], s2));
  return other & (far | (sumsq3_dev(m0, m1, m2) <= t.rcut2_hi));
}

// WM 0: count each atom's hits into cnt (and their maximum into *maxcnt); 1: emit them at
// off[i]..off[i+1]; 2: both at once, emitting into kcap padded slots per atom (i * kcap ..),
// hits beyond kcap dropped (the count and *maxcnt still see them).
template <int WM>
__global__ void __launch_bounds__(WALKC_WARPS * 32) k_pair_walk_cells(
    int64_t ncells, PairTest t, const ConfGrid* __restrict__ grid, const int32_t* __restrict__ conf,
    const int64_t* __restrict__ cell_start, const int32_t* __restrict__ cell_atoms, const double4* __restrict__ spos,
    int64_t* __restrict__ cnt, const int64_t* __restrict__ off, int32_t* __restrict__ outj,
    double* __restrict__ outr, int kcap, int* __restrict__ maxcnt) {
  constexpr bool EMIT = WM != 0;
  __shared__ WalkAtom sa[WALKC_WARPS][32];
  __shared__ WalkQ sq[WALKC_WARPS][WALK_RING];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t c = (int64_t)blockIdx.x * WALKC_WARPS + w;
  if (c >= ncells) return;  // warp-uniform; the kernel synchronises only within a warp
  const int64_t s0 = cell_start[c], s1 = cell_start[c + 1];
  if (s0 == s1) return;
  const ConfGrid g = grid[conf[cell_atoms[s0]]];
  int cc[3];
  {
    const double4 x0 = spos[s0];
    cell_coords(g, x0.x, x0.y, x0.z, cc);
  }
  StencilRanges R;
  stencil_ranges(g, cc, cell_start, R);
  const unsigned lt = (1u << lane) - 1u;
  WalkAtom* A = sa[w];
  WalkQ* Q = sq[w];
  for (int64_t g0 = s0; g0 < s1; g0 += 32) {
    const int G = (int)((s1 - g0) < 32 ? (s1 - g0) : 32);
    __syncwarp();
    if (lane < G) {
      const int32_t i = cell_atoms[g0 + lane];
      A[lane].i = i;
      A[lane].cnt = 0;
      A[lane].x = spos[g0 + lane];
      if (WM == 1) {
        A[lane].base = off[i];
        A[lane].end = off[i + 1];
      } else {
        A[lane].base = (int64_t)i * kcap;
        A[lane].end = (int64_t)i * kcap + kcap;
      }
    }
    __syncwarp();
    // the (range, chunk, atoms) sequence flattened, so that phase 2 has one call site: each
    // pass takes one step of phase 1, then drains full batches, and the remainder after the
    // last step
    int r = 0;
    while (r < R.n && R.beg[r] >= R.end[r]) r++;
    int64_t q0 = r < R.n ? R.beg[r] : 0, q = 0;
    int ii = 0;
    unsigned head = 0, tail = 0;  // ring positions (mod WALK_RING) of the first and next entries
    bool inq = false;
    int32_t j = 0;
    double4 xj = make_double4(0.0, 0.0, 0.0, 0.0);
    for (;;) {
      const bool more = r < R.n;  // warp-uniform
      if (more) {
        if (ii == 0) {  // a new chunk of candidates
          q = q0 + lane;
          inq = q < R.end[r];
          if (inq) {
            j = cell_atoms[q];
            xj = spos[q];
          }
        }
        bool cand[WALK_ILP];
#pragma unroll
        for (int k = 0; k < WALK_ILP; k++) {
          const int a = ii + k < G ? ii + k : ii;
          cand[k] = inq & (ii + k < G) & walk_prefilter(t, g.L, A[a].i, A[a].x, j, xj);
        }
#pragma unroll
        for (int k = 0; k < WALK_ILP; k++) {
          const unsigned bal = __ballot_sync(0xffffffffu, cand[k]);
          if (cand[k]) Q[(tail + __popc(bal & lt)) % WALK_RING] = WalkQ{(int32_t)q, ii + k};
          tail += __popc(bal);
        }
        ii += WALK_ILP;
        if (ii >= G) {
          ii = 0;
          q0 += 32;
          if (q0 >= R.end[r]) {
            do r++;
            while (r < R.n && R.beg[r] >= R.end[r]);
            if (r < R.n) q0 = R.beg[r];
          }
        }
      }
      while (tail - head >= 32u || (!more && tail != head)) {  // phase 2 on the next m queued pairs
        __syncwarp();
        const int m = tail - head < 32u ? (int)(tail - head) : 32;
        bool ok = false;
        int e_ii = 0;
        int32_t e_j = 0;
        double rr[3];
        if (lane < m) {
          const WalkQ e = Q[(head + lane) % WALK_RING];
          e_ii = e.ii;
          e_j = cell_atoms[e.slot];
          ok = pair_ok(t, g.L, A[e_ii].i, A[e_ii].x, e_j, spos[e.slot], rr);
        }
        const unsigned bal = __ballot_sync(0xffffffffu, ok);
        // lanes of the same atom: its members rank after the atom's running count
        const unsigned grp = __match_any_sync(0xffffffffu, lane < m ? e_ii : 32 + lane);
        if (EMIT && ok) {
          const int64_t o = A[e_ii].base + A[e_ii].cnt + __popc(bal & grp & lt);
          if (o < A[e_ii].end) {  // a list cut at the capacity (capacity mode) drops its tail
            outj[o] = e_j;
            outr[3 * o] = rr[0];
            outr[3 * o + 1] = rr[1];
            outr[3 * o + 2] = rr[2];
          }
        }
        __syncwarp();
        if (lane < m && (grp >> lane) == 1u) A[e_ii].cnt += __popc(bal & grp);  // the group's last lane
        head += m;
        __syncwarp();
      }
      if (!more) break;
    }
    if (WM != 1) {
      int km = 0;
      if (lane < G) {
        km = A[lane].cnt;
        cnt[A[lane].i] = km;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) km = max(km, __shfl_xor_sync(0xffffffffu, km, o));
      if (lane == 0) atomicMax(maxcnt, km);
    }
  }
}

// Capacity mode of the padded walk: an atom with more hits than slots is a capacity error.
__global__ void k_kcap_check(const int* __restrict__ maxcnt, int kcap, int* __restrict__ status) {
  if (threadIdx.x == 0 && *maxcnt > kcap) atomicExch(status, IPG_ERR_CAPACITY);
}

// Padded emission (k_pair_walk_cells<2>) to the CSR list: slot t of atom i goes to off[i] + t.
__global__ void k_pad_compact(int64_t n, int kcap, const int64_t* __restrict__ off, const int32_t* __restrict__ pj,
                              const double* __restrict__ pr, int32_t* __restrict__ j, double* __restrict__ r) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n * kcap) return;
  const int64_t i = s / kcap;
  const int64_t o = off[i] + (s - i * kcap);
  if (o >= off[i + 1]) return;
  j[o] = pj[s];
  r[3 * o] = pr[3 * s];
  r[3 * o + 1] = pr[3 * s + 1];
  r[3 * o + 2] = pr[3 * s + 2];
}

// Sorts each atom's list by neighbor index (insertion sort; lists are short).
__global__ void k_pair_sort(int64_t n, const int64_t* __restrict__ off, int32_t* __restrict__ j,
                            double* __restrict__ r) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t s = off[i], e = off[i + 1];
  for (int64_t a = s + 1; a < e; a++) {
    int32_t v = j[a];
    double r0 = r[3 * a], r1 = r[3 * a + 1], r2 = r[3 * a + 2];
    int64_t b = a - 1;
    while (b >= s && j[b] > v) {
      j[b + 1] = j[b];
      r[3 * (b + 1)] = r[3 * b];
      r[3 * (b + 1) + 1] = r[3 * b + 1];
      r[3 * (b + 1) + 2] = r[3 * b + 2];
      b--;
    }
    j[b + 1] = v;
    r[3 * (b + 1)] = r0;
    r[3 * (b + 1) + 1] = r1;
    r[3 * (b + 1) + 2] = r2;
  }
}

// Transpose: for every atom k, the pairs p whose neighbor is k, in ascending p.  The lists it
// serves (the full SNAP lists) are symmetric with one image per pair, so the pairs whose
// neighbor is k are those owned by k's own neighbors i, and ascending p is ascending i: pair
// (i -> k) takes slot #{q owned by k : j[q] < i} of k's in-list.  No atomics, no sort.  (A
// list cut at a capacity is not symmetric; its slots stay in bounds and the capacity error
// discards the result.)
__global__ void k_in_count(const int64_t* __restrict__ d_np, const int32_t* __restrict__ j,
                           int64_t* __restrict__ cnt) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= *d_np) return;
  atomicAdd((unsigned long long*)&cnt[j[p]], 1ull);
}
// One warp per owner i, one lane per pair (i -> k) (32 at a time); each lane counts the
// neighbors of k below i on its own, so the lanes' loads overlap.
__global__ void k_in_rank(int64_t n, const int64_t* __restrict__ off, const int32_t* __restrict__ j,
                          const int64_t* __restrict__ in_off, int64_t* __restrict__ in_pair) {
  const int lane = threadIdx.x & 31;
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= n) return;  // warp-uniform
  const int64_t p1 = off[i + 1];
  for (int64_t p = off[i] + lane; p < p1; p += 32) {
    const int32_t k = j[p];
    const int64_t q0 = off[k], q1 = off[k + 1];
    int64_t rank = 0;
#pragma unroll 4
    for (int64_t q = q0; q < q1; q++) rank += j[q] < i;
    const int64_t slot = in_off[k] + rank;
    if (slot < in_off[k + 1]) in_pair[slot] = p;
  }
}

inline unsigned nblk(int64_t n, int t) { return (unsigned)std::max<int64_t>(1, (n + t - 1) / t); }

}  // namespace

int ipg_build_cells(ipg_ctx* ctx, const char* prefix, int64_t n, const double* d_pos, const int32_t* d_species,
                    int nsp, int nconf, const int64_t* h_atom_off, const double* h_L, double radius, CellList& cl) {
  std::string pre(prefix);
  cl.nconf = nconf;
  cl.n = n;
  cl.radius = radius;
  cl.h_grid.assign(nconf, ConfGrid());
  bool any_open = false;
  for (int c = 0; c < nconf; c++) {
    ConfGrid& g = cl.h_grid[c];
    g.atom_off = h_atom_off[c];
    g.natoms = h_atom_off[c + 1] - h_atom_off[c];
    for (int a = 0; a < 3; a++) {
      double L = h_L[3 * c + a];
      if (!(L > 0.0)) return ipg_fail(ctx, IPG_ERR_ARG, "box length L[%d] of configuration %d must be > 0", a, c);
      g.L[a] = std::isinf(L) ? INFINITY : L;
      any_open |= std::isinf(L);
    }
  }
  IPG_RET(scratch(ctx, (pre + "grid").c_str(), nconf, &cl.d_grid));
  std::vector<double> ext(6 * (size_t)nconf, 0.0);
  if (any_open && n > 0 && ctx->capturing)
    return ipg_fail(ctx, IPG_ERR_UNSUPPORTED, "open boundaries cannot be captured in a graph");
  if (any_open && n > 0) {
    CUDA_RET(ctx, cudaMemcpyAsync(cl.d_grid, cl.h_grid.data(), sizeof(ConfGrid) * nconf, cudaMemcpyHostToDevice,
                                  ctx->stream));
    double* d_ext;
    IPG_RET(scratch(ctx, (pre + "ext").c_str(), 6 * (size_t)nconf, &d_ext));
    IPG_LAUNCH(ctx, k_extent, nconf, 256, 0, d_pos, cl.d_grid, d_ext);
    CUDA_RET(ctx, cudaMemcpyAsync(ext.data(), d_ext, sizeof(double) * 6 * nconf, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_RET(ctx, cudaStreamSynchronize(ctx->stream));
  }
  const double rc = radius * (1.0 + 1e-9);
  int64_t cell_total = 0;
  for (int c = 0; c < nconf; c++) {
    ConfGrid& g = cl.h_grid[c];
    int64_t tot = 1;
    double e3[3];
    for (int a = 0; a < 3; a++) {
      double lo = 0.0, e = g.L[a];
      if (std::isinf(g.L[a])) {
        lo = ext[6 * c + a];
        e = ext[6 * c + 3 + a] - lo;
        if (!(e >= 0.0) || !std::isfinite(e)) {  // empty config or non-finite input
          lo = 0.0;
          e = 0.0;
        }
      }
      g.lo[a] = lo;
      e3[a] = e;
      int nc = 1;
      if (rc > 0.0 && std::isfinite(rc) && e > 0.0) nc = (int)std::max(1.0, std::min(std::floor(e / rc), 1024.0));
      g.nc[a] = nc;
      tot *= nc;
    }
    while (tot > std::max<int64_t>(64, 8 * g.natoms)) {  // keep the grid proportional to the atoms
      int a = (g.nc[0] >= g.nc[1] && g.nc[0] >= g.nc[2]) ? 0 : (g.nc[1] >= g.nc[2] ? 1 : 2);
      tot /= g.nc[a];
      g.nc[a] = std::max(1, g.nc[a] / 2);
      tot *= g.nc[a];
    }
    for (int a = 0; a < 3; a++) g.cs[a] = e3[a] > 0.0 ? e3[a] / g.nc[a] : 1.0;
    g.cell_off = cell_total;
    cell_total += tot;
  }
  if (cell_total >= (int64_t)INT32_MAX) return ipg_fail(ctx, IPG_ERR_CAPACITY, "too many cells");
  cl.ncells = cell_total;
  if (!ctx->capturing)  // a captured graph's grid table is uploaded before each replay
    CUDA_RET(ctx, cudaMemcpyAsync(cl.d_grid, cl.h_grid.data(), sizeof(ConfGrid) * nconf, cudaMemcpyHostToDevice,
                                  ctx->stream));
  int64_t *count, *fill;
  int32_t* cell_of;
  IPG_RET(scratch(ctx, (pre + "conf").c_str(), n, &cl.d_conf));
  IPG_RET(scratch(ctx, (pre + "cell_of").c_str(), n, &cell_of));
  IPG_RET(scratch(ctx, (pre + "cell_start").c_str(), cell_total + 1, &cl.d_cell_start));
  IPG_RET(scratch(ctx, (pre + "cell_fill").c_str(), cell_total + 1, &fill));
  IPG_RET(scratch(ctx, (pre + "cell_atoms").c_str(), n, &cl.d_cell_atoms));
  IPG_RET(scratch(ctx, (pre + "slot_of").c_str(), n, &cl.d_slot_of));
  IPG_RET(scratch(ctx, (pre + "spos").c_str(), n, &cl.d_spos));
  count = cl.d_cell_start;
  CUDA_RET(ctx, cudaMemsetAsync(count, 0, sizeof(int64_t) * (cell_total + 1), ctx->stream));
  CUDA_RET(ctx, cudaMemsetAsync(fill, 0, sizeof(int64_t) * (cell_total + 1), ctx->stream));
  if (n == 0) return IPG_OK;
  IPG_LAUNCH(ctx, k_cell_count, nblk(n, 256), 256, 0, n, d_pos, d_species, nsp, cl.d_grid, nconf, cl.d_conf, cell_of,
             count, ctx->d_status);
  IPG_RET(ipg_scan_i64(ctx, count, cl.d_cell_start, cell_total + 1));
  IPG_LAUNCH(ctx, k_cell_fill, nblk(n, 256), 256, 0, n, cell_of, cl.d_cell_start, fill, cl.d_cell_atoms);
  IPG_LAUNCH(ctx, k_cell_sort, nblk(cell_total, 128), 128, 0, cell_total, cl.d_cell_start, cl.d_cell_atoms);
  IPG_LAUNCH(ctx, k_cell_gather, nblk(n, 256), 256, 0, n, cl.d_cell_atoms, d_pos, d_species, nsp, cl.d_slot_of,
             cl.d_spos);
  return IPG_OK;
}

namespace {
// The in-lists of a symmetric list (k_in_rank): in_off by counting, in_pair by rank.
int build_transpose(ipg_ctx* ctx, const std::string& pre, int64_t n, PairList& pl) {
  IPG_RET(scratch(ctx, (pre + "in_off").c_str(), n + 1, &pl.d_in_off));
  IPG_RET(scratch(ctx, (pre + "in_pair").c_str(), pl.npairs + 1, &pl.d_in_pair));
  CUDA_RET(ctx, cudaMemsetAsync(pl.d_in_off, 0, sizeof(int64_t) * (n + 1), ctx->stream));
  if (pl.npairs > 0) IPG_LAUNCH(ctx, k_in_count, nblk(pl.npairs, 256), 256, 0, pl.d_np, pl.d_j, pl.d_in_off);
  IPG_RET(ipg_scan_i64(ctx, pl.d_in_off, pl.d_in_off, n + 1));
  if (pl.npairs > 0)
    IPG_LAUNCH(ctx, k_in_rank, nblk(32 * n, 128), 128, 0, n, pl.d_off, pl.d_j, pl.d_in_off, pl.d_in_pair);
  return IPG_OK;
}
}  // namespace

int ipg_build_pairs(ipg_ctx* ctx, const char* prefix, const CellList& cl, const int32_t* d_species, int nsp,
                    const double* h_cut, int mode, bool want_transpose, PairList& pl, bool sorted, int64_t cap,
                    int walk_warps, bool count_only) {
  const int wt = 32 * std::max(1, std::min(4, walk_warps));
  (void)d_species;
  IPG_RET(ipg_side_join(ctx));
  std::string pre(prefix);
  PairTest t;
  memset(&t, 0, sizeof(t));
  t.mode = mode & 0xff;
  t.literal = (mode & IPG_NLIST_LITERAL_SQRT) ? 1 : 0;
  t.nsp = nsp;
  if (t.mode == IPG_NLIST_HALF) {
    t.rcut = h_cut[0];
  } else {
    if (nsp < 1 || nsp > 8) return ipg_fail(ctx, IPG_ERR_ARG, "nspecies must be in 1..8 for a full list");
    double cutmax2 = 0.0;
    for (int q = 0; q < nsp * nsp; q++) {
      t.cutsq[q] = h_cut[q];
      cutmax2 = std::max(cutmax2, h_cut[q]);
    }
    double cutmax = std::sqrt(cutmax2);
    t.rcut = t.literal ? std::sqrt(cutmax) : cutmax;
  }
  t.rcut2_lo = t.rcut * t.rcut * (1.0 - 1e-12);
  t.rcut2_hi = t.rcut * t.rcut * (1.0 + 1e-12);
  int64_t n = cl.n;
  pl.n = n;
  int64_t* cnt;
  IPG_RET(scratch(ctx, (pre + "off").c_str(), n + 1, &pl.d_off));
  cnt = pl.d_off;
  CUDA_RET(ctx, cudaMemsetAsync(cnt, 0, sizeof(int64_t) * (n + 1), ctx->stream));
  const bool by_cell = ctx->walk_by_cell;
  // One walk instead of two when a previous build of this list gave the per-atom maximum:
  // emit into padded slots while counting, then compact (or, if an atom overflowed its
  // slots, emit again at the counted offsets).  In capacity mode (graph capture) there is no
  // read-back: an overflow sets IPG_ERR_CAPACITY in the device status word instead.
  int* maxcnt;
  IPG_RET(scratch(ctx, (pre + "maxcnt").c_str(), 1, &maxcnt));
  CUDA_RET(ctx, cudaMemsetAsync(maxcnt, 0, sizeof(int), ctx->stream));
  int kcap = (by_cell && !count_only && ctx->walk_single) ? ctx->walk_kcap[pre] : 0;
  if ((double)n * kcap * 28.0 > 2.0 * (1 << 30)) kcap = 0;  // padded slots within 2 GiB
  int32_t* pad_j = nullptr;
  double* pad_r = nullptr;
  if (kcap > 0 && n > 0) {
    IPG_RET(scratch(ctx, (pre + "pad_j").c_str(), (size_t)n * kcap + 1, &pad_j));
    IPG_RET(scratch(ctx, (pre + "pad_r").c_str(), 3 * (size_t)n * kcap + 3, &pad_r));
  }
  if (n > 0) {
    if (by_cell && kcap > 0)
      IPG_LAUNCH(ctx, k_pair_walk_cells<2>, nblk(cl.ncells, WALKC_WARPS), WALKC_WARPS * 32, 0, cl.ncells, t,
                 cl.d_grid, cl.d_conf, cl.d_cell_start, cl.d_cell_atoms, cl.d_spos, cnt, nullptr, pad_j, pad_r, kcap,
                 maxcnt);
    else if (by_cell)
      IPG_LAUNCH(ctx, k_pair_walk_cells<0>, nblk(cl.ncells, WALKC_WARPS), WALKC_WARPS * 32, 0, cl.ncells, t,
                 cl.d_grid, cl.d_conf, cl.d_cell_start, cl.d_cell_atoms, cl.d_spos, cnt, nullptr, nullptr, nullptr, 0,
                 maxcnt);
    else
      IPG_LAUNCH(ctx, k_pair_walk<false>, nblk(32 * n, wt), wt, 0, n, t, cl.d_grid, cl.d_conf, cl.d_cell_start,
                 cl.d_cell_atoms, cl.d_spos, cnt, nullptr, nullptr, nullptr);
  }
  IPG_RET(ipg_scan_i64(ctx, cnt, pl.d_off, n + 1));
  pl.d_np = pl.d_off + n;
  int hmax = 0;
  if (cap > 0) {  // capacity mode: no read-back
    pl.npairs = cap;
    IPG_LAUNCH(ctx, k_clamp_offsets, nblk(n + 1, 256), 256, 0, n, pl.d_off, cap, ctx->d_status);
    if (kcap > 0 && n > 0) IPG_LAUNCH(ctx, k_kcap_check, 1, 32, 0, maxcnt, kcap, ctx->d_status);
  } else {
    CUDA_RET(ctx, cudaMemcpyAsync(&pl.npairs, pl.d_off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_RET(ctx, cudaMemcpyAsync(&hmax, maxcnt, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_RET(ctx, cudaStreamSynchronize(ctx->stream));
    if (by_cell && !count_only) ctx->walk_kcap[pre] = ((hmax + hmax / 8 + 4 + 7) / 8) * 8;  // next build
  }
  if (pl.npairs >= (int64_t)1 << 40) return ipg_fail(ctx, IPG_ERR_CAPACITY, "pair count overflow");
  if (count_only) return IPG_OK;
  IPG_RET(scratch(ctx, (pre + "j").c_str(), pl.npairs + 1, &pl.d_j));
  IPG_RET(scratch(ctx, (pre + "r").c_str(), 3 * pl.npairs + 3, &pl.d_r));
  if (n > 0) {
    if (by_cell && kcap > 0 && (cap > 0 || hmax <= kcap))
      IPG_LAUNCH(ctx, k_pad_compact, nblk(n * kcap, 256), 256, 0, n, kcap, pl.d_off, pad_j, pad_r, pl.d_j, pl.d_r);
    else if (by_cell)
      IPG_LAUNCH(ctx, k_pair_walk_cells<1>, nblk(cl.ncells, WALKC_WARPS), WALKC_WARPS * 32, 0, cl.ncells, t,
                 cl.d_grid, cl.d_conf, cl.d_cell_start, cl.d_cell_atoms, cl.d_spos, nullptr, pl.d_off, pl.d_j,
                 pl.d_r, 0, nullptr);
    else
      IPG_LAUNCH(ctx, k_pair_walk<true>, nblk(32 * n, wt), wt, 0, n, t, cl.d_grid, cl.d_conf, cl.d_cell_start,
                 cl.d_cell_atoms, cl.d_spos, nullptr, pl.d_off, pl.d_j, pl.d_r);
    if (sorted) IPG_LAUNCH(ctx, k_pair_sort, nblk(n, 128), 128, 0, n, pl.d_off, pl.d_j, pl.d_r);
  }
  if (want_transpose) {
    // needed only by the force gather: for one configuration it overlaps the first SNAP
    // kernels on the side stream (+0.6% at 54,000 atoms); for a batch the overlap measured
    // 2.6% slower (512 configurations), so batches build it in order
    const bool side = cl.nconf == 1;
    if (side) IPG_RET(ipg_side_begin(ctx));
    const int st = build_transpose(ctx, pre, n, pl);
    if (side) IPG_RET(ipg_side_end(ctx));
    IPG_RET(st);
  }
  return IPG_OK;
}

int ipg_max_disp2(ipg_ctx* ctx, const CellList& cl, const double* d_pos, const double* d_ref,
                  const int32_t* d_species, const int32_t* d_ref_species, double* out) {
  *out = 0.0;
  if (cl.n == 0) return IPG_OK;
  unsigned long long* d_m;
  IPG_RET(scratch(ctx, "skin_maxdisp", 1, &d_m));
  CUDA_RET(ctx, cudaMemsetAsync(d_m, 0, sizeof(unsigned long long), ctx->stream));
  const int64_t grid = std::min<int64_t>(nblk(cl.n, 256), 4 * ctx->num_sms);
  IPG_LAUNCH(ctx, k_max_disp2, (unsigned)grid, 256, 0, cl.n, cl.d_grid, cl.d_conf, d_pos, d_ref, d_species,
             d_ref_species, d_m);
  unsigned long long h = 0;
  CUDA_RET(ctx, cudaMemcpyAsync(&h, d_m, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_RET(ctx, cudaStreamSynchronize(ctx->stream));
  memcpy(out, &h, sizeof(double));
  return IPG_OK;
}

int ipg_filter_pairs(ipg_ctx* ctx, const char* prefix, const CellList& cl, const PairList& cached,
                     const double* d_pos, const int32_t* d_species, int nsp, const double* h_cut, int mode,
                     PairList& pl) {
  IPG_RET(ipg_side_join(ctx));
  std::string pre(prefix);
  PairTest t;
  memset(&t, 0, sizeof(t));
  t.mode = IPG_NLIST_FULL;
  t.literal = (mode & IPG_NLIST_LITERAL_SQRT) ? 1 : 0;
  t.nsp = nsp;
  double cutmax2 = 0.0;
  for (int q = 0; q < nsp * nsp; q++) {
    t.cutsq[q] = h_cut[q];
    cutmax2 = std::max(cutmax2, h_cut[q]);
  }
  const double cutmax = std::sqrt(cutmax2);
  t.rcut = t.literal ? std::sqrt(cutmax) : cutmax;
  t.rcut2_lo = t.rcut * t.rcut * (1.0 - 1e-12);
  t.rcut2_hi = t.rcut * t.rcut * (1.0 + 1e-12);
  const int64_t n = cl.n;
  pl.n = n;
  IPG_RET(scratch(ctx, (pre + "off").c_str(), n + 1, &pl.d_off));
  CUDA_RET(ctx, cudaMemsetAsync(pl.d_off, 0, sizeof(int64_t) * (n + 1), ctx->stream));
  if (n > 0)
    IPG_LAUNCH(ctx, k_filter_walk<false>, nblk(32 * n, 128), 128, 0, n, t, cl.d_grid, cl.d_conf, cached.d_off,
               cached.d_j, d_pos, d_species, nsp, pl.d_off, nullptr, nullptr, nullptr, ctx->d_status);
  IPG_RET(ipg_scan_i64(ctx, pl.d_off, pl.d_off, n + 1));
  pl.d_np = pl.d_off + n;
  CUDA_RET(ctx, cudaMemcpyAsync(&pl.npairs, pl.d_off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_RET(ctx, cudaStreamSynchronize(ctx->stream));
  IPG_RET(scratch(ctx, (pre + "j").c_str(), pl.npairs + 1, &pl.d_j));
  IPG_RET(scratch(ctx, (pre + "r").c_str(), 3 * pl.npairs + 3, &pl.d_r));
  if (n > 0)
    IPG_LAUNCH(ctx, k_filter_walk<true>, nblk(32 * n, 128), 128, 0, n, t, cl.d_grid, cl.d_conf, cached.d_off,
               cached.d_j, d_pos, d_species, nsp, nullptr, pl.d_off, pl.d_j, pl.d_r, ctx->d_status);
  const bool side = cl.nconf == 1;  // as in ipg_build_pairs
  if (side) IPG_RET(ipg_side_begin(ctx));
  const int st = build_transpose(ctx, pre, n, pl);
  if (side) IPG_RET(ipg_side_end(ctx));
  IPG_RET(st);
  return IPG_OK;
}

// ---------------------------------------------------------------------------------
struct ipg_nlist {
  int64_t n = 0, npairs = 0;
  std::vector<int64_t> off;
  std::vector<int32_t> j;
  std::vector<double> r;
};

namespace {

// Validates and uploads the inputs and builds the pair list (or only counts it).
int neighbor_pairs(ipg_ctx* ctx, int64_t n, const double* pos, const double L[3], const int32_t* species,
                   int32_t nspecies, const double* cut, int32_t mode, bool count_only, PairList& pl) {
  if (!ctx || n < 0 || (n > 0 && !pos) || !L || !cut) return IPG_ERR_ARG;
  if (n >= INT32_MAX) return ipg_fail(ctx, IPG_ERR_ARG, "n too large");
  int base = mode & 0xff;
  if (base != IPG_NLIST_HALF && base != IPG_NLIST_FULL) return ipg_fail(ctx, IPG_ERR_ARG, "bad mode");
  if (base == IPG_NLIST_FULL && !species) return ipg_fail(ctx, IPG_ERR_ARG, "full list needs species");
  CUDA_RET(ctx, cudaSetDevice(ctx->device));
  if (!host_all_finite(pos, 3 * n)) return ipg_fail(ctx, IPG_ERR_NONFINITE, "non-finite position");
  if (species && !host_species_ok(species, n, std::max(1, (int)nspecies)))
    return ipg_fail(ctx, IPG_ERR_SPECIES, "species id out of range");
  double *d_pos;
  int32_t* d_sp = nullptr;
  IPG_RET(scratch(ctx, "nl_in_pos", 3 * (size_t)n + 3, &d_pos));
  if (n) CUDA_RET(ctx, cudaMemcpyAsync(d_pos, pos, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, ctx->stream));
  if (species) {
    IPG_RET(scratch(ctx, "nl_in_sp", (size_t)n + 1, &d_sp));
    if (n) CUDA_RET(ctx, cudaMemcpyAsync(d_sp, species, sizeof(int32_t) * n, cudaMemcpyHostToDevice, ctx->stream));
  }
  IPG_RET(ipg_status_reset(ctx));
  int64_t aoff[2] = {0, n};
  double radius;
  if (base == IPG_NLIST_HALF) {
    radius = cut[0];
  } else {
    double m = 0.0;
    for (int q = 0; q < nspecies * nspecies; q++) m = std::max(m, cut[q]);
    radius = std::sqrt(m);
    if (mode & IPG_NLIST_LITERAL_SQRT) radius = std::sqrt(radius);
  }
  if (!(radius >= 0.0)) return ipg_fail(ctx, IPG_ERR_ARG, "cutoff must be >= 0");
  CellList cl;
  IPG_RET(ipg_build_cells(ctx, "nl_", n, d_pos, d_sp, std::max(1, (int)nspecies), 1, aoff, L, radius, cl));
  IPG_RET(ipg_build_pairs(ctx, "nl_", cl, d_sp, std::max(1, (int)nspecies), cut, mode, false, pl, true, 0, 4,
                          count_only));
  return ipg_status_check(ctx, count_only ? "ipg_neighbor_count" : "ipg_neighbor_build");
}

}  // namespace

extern "C" {

int ipg_neighbor_count(ipg_ctx* ctx, int64_t n, const double* pos, const double L[3], const int32_t* species,
                       int32_t nspecies, const double* cut, int32_t mode, int64_t* npairs) {
  if (!npairs) return IPG_ERR_ARG;
  PairList pl;
  IPG_RET(neighbor_pairs(ctx, n, pos, L, species, nspecies, cut, mode, true, pl));
  *npairs = pl.npairs;
  return IPG_OK;
}

int ipg_neighbor_build(ipg_ctx* ctx, int64_t n, const double* pos, const double L[3], const int32_t* species,
                       int32_t nspecies, const double* cut, int32_t mode, ipg_nlist** out) {
  if (!out) return IPG_ERR_ARG;
  PairList pl;
  IPG_RET(neighbor_pairs(ctx, n, pos, L, species, nspecies, cut, mode, false, pl));
  ipg_nlist* nl = new ipg_nlist();
  nl->n = n;
  nl->npairs = pl.npairs;
  nl->off.resize(n + 1);
  nl->j.resize(pl.npairs);
  nl->r.resize(3 * pl.npairs);
  CUDA_RET(ctx, cudaMemcpyAsync(nl->off.data(), pl.d_off, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost,
                                ctx->stream));
  if (pl.npairs) {
    CUDA_RET(ctx, cudaMemcpyAsync(nl->j.data(), pl.d_j, sizeof(int32_t) * pl.npairs, cudaMemcpyDeviceToHost,
                                  ctx->stream));
    CUDA_RET(ctx, cudaMemcpyAsync(nl->r.data(), pl.d_r, sizeof(double) * 3 * pl.npairs, cudaMemcpyDeviceToHost,
                                  ctx->stream));
  }
  int st = ipg_sync(ctx);
  if (st) {
    delete nl;
    return st;
  }
  *out = nl;
  return IPG_OK;
}

int ipg_nlist_size(const ipg_nlist* nl, int64_t* npairs) {
  if (!nl || !npairs) return IPG_ERR_ARG;
  *npairs = nl->npairs;
  return IPG_OK;
}

int ipg_nlist_export(const ipg_nlist* nl, int64_t* offsets, int32_t* j, double* r) {
  if (!nl) return IPG_ERR_ARG;
  if (offsets) memcpy(offsets, nl->off.data(), sizeof(int64_t) * (nl->n + 1));
  if (j && nl->npairs) memcpy(j, nl->j.data(), sizeof(int32_t) * nl->npairs);
  if (r && nl->npairs) memcpy(r, nl->r.data(), sizeof(double) * 3 * nl->npairs);
  return IPG_OK;
}

int ipg_nlist_free(ipg_nlist* nl) {
  if (!nl) return IPG_ERR_ARG;
  delete nl;
  return IPG_OK;
}

}  // extern "C"
