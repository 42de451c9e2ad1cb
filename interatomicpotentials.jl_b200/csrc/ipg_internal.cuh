// ipg_internal.cuh — shared definitions of the libipg CUDA sources (sm_100a, FP64).
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "ipg.h"

// ----------------------------------------------------------------------------------
// Context: one CUDA stream, named growable device scratch buffers, a device status
// word that kernels raise instead of trapping, and the last error message.
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
};

struct ipg_ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  std::string err;
  int64_t launches = 0;
  int* d_status = nullptr;  // device status word (IPG_OK or a negative code)
  int* h_status = nullptr;  // pinned mirror
  std::map<std::string, DevBuf> bufs;
  std::map<std::string, std::vector<char>> hbufs;
  // optional per-kernel device timing (ipg_timing_enable / ipg_timing_read)
  bool timing = false;
  struct Timed {
    std::vector<cudaEvent_t> ev;  // start/stop pairs
    double ms = 0.0;
    int64_t launches = 0;
  };
  std::map<std::string, Timed> timed;
  std::vector<cudaEvent_t> event_pool;
  // CUDA-graph capture: while capturing, scratch buffers must not move (an allocation
  // fails the capture) and host tables are not re-uploaded (the replay path uploads them
  // before each launch).  scratch_gen counts (re)allocations: a graph whose generation
  // differs refers to freed buffers and is discarded.
  bool capturing = false;
  uint64_t scratch_gen = 0;
  bool walk_by_cell = true;  // neighbor walk: one warp per cell (false: one warp per atom)
  bool pair_full_stencil = false;  // pair potentials: full-stencil walk even where the half stencil applies
  int pair_minb = 3;               // pair potentials: register bound of the half-stencil kernel (3, 4, 5)
  // single-pass neighbor walk: per list prefix, the per-atom slot count of the padded
  // emission (from the largest count of the previous build; 0 = walk twice)
  std::map<std::string, int> walk_kcap;
  bool walk_single = true;
  // side stream for work that only a later kernel needs (the list transpose): forked from and
  // joined back into `stream` by events, so it also works inside a graph capture
  cudaStream_t side = nullptr;
  cudaStream_t side_main = nullptr;  // `stream` while the side stream stands in for it
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool side_pending = false;
  bool side_enabled = true;  // IPG_SIDE_STREAM=0: everything on `stream`
  // pinned staging ring for large copies between device memory and the caller's pageable host
  // buffers (ipg_copy_d2h / ipg_copy_h2d), and the host threads that split each slot's memcpy
  static constexpr int PIN_SLOTS = 4;
  char* pinned[PIN_SLOTS] = {};
  cudaEvent_t pinned_ev[PIN_SLOTS] = {};
  struct HostCopyTeam* copy_team = nullptr;
  int copy_threads = 0;  // threads per host memcpy, the caller included (0: chosen at first use)
  // CUDA graphs of ipg_pair_eval_dev (IPG_PAIR_GRAPH), keyed by the call's inputs
  struct PairGraph {
    int64_t n = 0;
    double L[3] = {0, 0, 0};
    const void *pos = nullptr, *sp = nullptr, *E = nullptr, *F = nullptr, *W6 = nullptr;
    uint32_t flags = 0;
    std::vector<char> terms;        // the ipg_pair_term array, bytewise
    std::vector<char> grid;         // the cell grid (ConfGrid) the replay uploads
    int full_stencil = 0, minb = 0;
    cudaGraphExec_t exec = nullptr;
    uint64_t gen = 0;               // scratch generation at capture
  };
  std::vector<PairGraph> pair_graphs;
  int64_t pair_graph_replays = 0;
};

constexpr int IPG_ERR_NOT_CAPTURED = 1;  // internal: no CUDA graph for this key (not an API code)

// Runs the launches between ipg_side_begin and ipg_side_end on the side stream (ctx->stream
// points at it meanwhile), after everything already on the main stream; ipg_side_join makes
// the main stream wait for them.  ipg_status_check and the list builders join first.
int ipg_side_begin(ipg_ctx* ctx);
int ipg_side_end(ipg_ctx* ctx);
int ipg_side_join(ipg_ctx* ctx);

// Records a start/stop event pair around a launch when timing is enabled.
int ipg_timing_mark(ipg_ctx* ctx, const char* name, bool start);

// Status propagation: every internal function returns int.
#define IPG_RET(x)            \
  do {                        \
    int _st = (x);            \
    if (_st != IPG_OK) return _st; \
  } while (0)

int ipg_fail(ipg_ctx* ctx, int code, const char* fmt, ...);

// Host input checks as single branch-free passes (the compiler vectorises them; the early-exit
// loops they replace cost ~0.1 ms per 54,000 atoms in front of every host-pointer call).
inline bool host_all_finite(const double* x, int64_t m) {
  uint64_t bad = 0;
  for (int64_t k = 0; k < m; k++) {
    uint64_t b;
    memcpy(&b, x + k, sizeof(b));
    bad |= (uint64_t)(((b >> 52) & 0x7ffu) == 0x7ffu);  // exponent all ones: Inf or NaN
  }
  return bad == 0;
}
inline bool host_species_ok(const int32_t* sp, int64_t n, int nsp) {
  uint32_t bad = 0;
  for (int64_t k = 0; k < n; k++) bad |= (uint32_t)((uint32_t)sp[k] >= (uint32_t)nsp);
  return bad == 0;
}
int ipg_cuda_check(ipg_ctx* ctx, cudaError_t e, const char* what);

#define CUDA_RET(ctx, call) IPG_RET(ipg_cuda_check((ctx), (call), #call))

// Named device scratch: grows (never shrinks) to at least `bytes`.
int ipg_scratch(ipg_ctx* ctx, const char* name, size_t bytes, void** out);
template <class T>
int scratch(ipg_ctx* ctx, const char* name, size_t count, T** out) {
  void* p = nullptr;
  IPG_RET(ipg_scratch(ctx, name, count * sizeof(T) + 16, &p));
  *out = static_cast<T*>(p);
  return IPG_OK;
}
// Named host staging buffer (pageable: for small uploads, which the driver copies out of the
// buffer before cudaMemcpyAsync returns).
template <class T>
T* host_scratch(ipg_ctx* ctx, const char* name, size_t count) {
  auto& v = ctx->hbufs[name];
  if (v.size() < count * sizeof(T)) v.resize(count * sizeof(T));
  return reinterpret_cast<T*>(v.data());
}

// Copies between device memory and a caller's (pageable) host buffer on ctx->stream.  Large
// copies go through a ring of four pinned chunks, so the DMAs of some chunks overlap the host
// copy of another, and each chunk's host copy is split over a team of host threads; a copy
// from pageable memory is staged by the driver at a fraction of the bandwidth.  ipg_copy_d2h returns once `dst` holds the data (it synchronises with the stream);
// ipg_copy_h2d returns once `src` may be reused.
int ipg_copy_d2h(ipg_ctx* ctx, void* dst, const void* src, size_t bytes);
int ipg_copy_h2d(ipg_ctx* ctx, void* dst, const void* src, size_t bytes);
// Joins the host copy threads (ipg_ctx_destroy).
void ipg_copy_team_free(ipg_ctx* ctx);

// Kernel launch with accounting and error check.
#define IPG_LAUNCH(ctx, kernel, grid, block, smem, ...)                                          \
  do {                                                                                           \
    kernel<<<(grid), (block), (smem), (ctx)->stream>>>(__VA_ARGS__);                             \
    (ctx)->launches++;                                                                           \
    IPG_RET(ipg_cuda_check((ctx), cudaGetLastError(), #kernel));                                 \
  } while (0)

// As IPG_LAUNCH, bracketed by timing events named `name` when timing is enabled.
#define IPG_TIMED_LAUNCH(ctx, name, kernel, grid, block, smem, ...) \
  do {                                                             \
    IPG_RET(ipg_timing_mark((ctx), (name), true));                 \
    IPG_LAUNCH(ctx, kernel, grid, block, smem, __VA_ARGS__);       \
    IPG_RET(ipg_timing_mark((ctx), (name), false));                \
  } while (0)

// Resets the device status word (async) and reads it back after a sync.
int ipg_status_reset(ipg_ctx* ctx);
int ipg_status_check(ipg_ctx* ctx, const char* what);
int ipg_sync(ipg_ctx* ctx);

// Exclusive scan of n+1 int64 values (in[n] must be 0): out[k] = sum_{q<k} in[q];
// out[n] is the total.  `out` may alias `in`.
int ipg_scan_i64(ipg_ctx* ctx, const int64_t* in, int64_t* out, int64_t n_plus_1);

// Sets device status to `code` (first error wins).
__device__ __forceinline__ void dev_raise(int* status, int code) { atomicCAS(status, 0, code); }

// ----------------------------------------------------------------------------------
// Minimum-image arithmetic of the reference, reproduced bit for bit (no FMA contraction).
// Julia mod(x, y) for y > 0 finite (the sign of the result follows y).
__device__ __forceinline__ double jl_mod_dev(double x, double L) {
  double r = (fabs(x) < L) ? x : fmod(x, L);  // fmod(x, L) == x exactly when |x| < L
  if (r == 0.0) return 0.0;
  if (r < 0.0) r = __dadd_rn(r, L);
  return r;
}
// src/nnlist.jl:18-21 get_displacement (one axis); L = +inf marks an open axis.
__device__ __forceinline__ double disp_axis_dev(double L, double x, double y) {
  double dx = __dsub_rn(x, y);
  if (isinf(L)) return dx;
  double d = jl_mod_dev(dx, L);
  return (__dmul_rn(2.0, d) < L) ? d : __dsub_rn(d, L);
}
// Distances.jl PeriodicEuclidean, one axis: min(mod(|a-b|, L), L - mod(|a-b|, L)).
__device__ __forceinline__ double pe_axis_dev(double L, double a, double b) {
  double s1 = fabs(__dsub_rn(a, b));
  if (isinf(L)) return s1;
  double s2 = (s1 < L) ? s1 : fmod(s1, L);
  double s3 = __dsub_rn(L, s2);
  return s2 < s3 ? s2 : s3;
}
__device__ __forceinline__ double sumsq3_dev(double a, double b, double c) {
  return __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c));
}

// ----------------------------------------------------------------------------------
// Cell lists (ipg_nlist.cu).  Configurations are independent boxes; atoms of config c are
// [atom_off[c], atom_off[c+1]).  Each configuration owns its own cell grid.
struct ConfGrid {
  double L[3];   // box diagonal, +inf on open axes
  double lo[3];  // grid origin
  double cs[3];  // cell edge (>= search radius on every axis with more than one cell)
  int nc[3];     // cells per axis
  int pad;
  int64_t cell_off;  // first global cell id of this configuration
  int64_t atom_off;
  int64_t natoms;
};

struct CellList {
  int nconf = 0;
  int64_t n = 0;
  int64_t ncells = 0;
  double radius = 0.0;
  ConfGrid* d_grid = nullptr;      // [nconf]
  std::vector<ConfGrid> h_grid;    // host copy
  int32_t* d_conf = nullptr;       // [n] configuration of each atom
  int64_t* d_cell_start = nullptr; // [ncells+1]
  int32_t* d_cell_atoms = nullptr; // [n] atom ids in cell order (ascending inside a cell)
  int32_t* d_slot_of = nullptr;    // [n] slot of each atom
  double4* d_spos = nullptr;       // [n] positions in slot order (w = species as double)
};

// Builds the cell list for `radius` (prefix selects the scratch buffers used).
// Species ids outside [0, nsp) raise IPG_ERR_SPECIES in the device status word.
int ipg_build_cells(ipg_ctx* ctx, const char* prefix, int64_t n, const double* d_pos, const int32_t* d_species,
                    int nsp, int nconf, const int64_t* h_atom_off, const double* h_L, double radius, CellList& cl);

// Materialised pair list in CSR form over atoms (original order), neighbors ascending.
struct PairList {
  int64_t n = 0;
  int64_t npairs = 0;        // exact count, or the capacity in capacity mode (buffer sizes, grids)
  const int64_t* d_np = nullptr;  // device copy of the count (d_off + n): what pair kernels read
  int64_t* d_off = nullptr;  // [n+1]
  int32_t* d_j = nullptr;    // [npairs]
  double* d_r = nullptr;     // [npairs][3]
  int64_t* d_in_off = nullptr;  // [n+1]   transpose: pairs whose neighbor is atom k
  int64_t* d_in_pair = nullptr; // [npairs]
};

// mode: IPG_NLIST_HALF (cut[0] = rcut) or IPG_NLIST_FULL (cut = nsp*nsp cutsq), with
// IPG_NLIST_LITERAL_SQRT optionally or-ed in.  want_transpose builds d_in_off/d_in_pair.
// sorted: each atom's neighbors ascending (the reference's order); otherwise the
// emission order (stencil cells in fixed order, ascending inside a cell), which is
// equally deterministic.
// cap > 0 selects capacity mode (no host read-back, so the build can be captured in a CUDA
// graph): buffers hold cap pairs; a larger count sets IPG_ERR_CAPACITY in the status word
// and every atom's list is cut at cap, so later kernels stay in bounds.
// Verlet-skin reuse: pl = the pairs of `cached` (a full list built with enlarged cutoffs over
// the cell list cl) that pass the true full-list test at d_pos, with their transpose.
int ipg_filter_pairs(ipg_ctx* ctx, const char* prefix, const CellList& cl, const PairList& cached,
                     const double* d_pos, const int32_t* d_species, int nsp, const double* h_cut, int mode,
                     PairList& pl);
// Largest squared minimum-image displacement of d_pos from d_ref (host value, synchronises);
// +inf when a position is not finite or a species id differs from d_ref_species.
int ipg_max_disp2(ipg_ctx* ctx, const CellList& cl, const double* d_pos, const double* d_ref,
                  const int32_t* d_species, const int32_t* d_ref_species, double* out);
// walk_warps: atoms (warps) per block of the neighbor walk, 1..4.
int ipg_build_pairs(ipg_ctx* ctx, const char* prefix, const CellList& cl, const int32_t* d_species, int nsp,
                    const double* h_cut, int mode, bool want_transpose, PairList& pl, bool sorted = true,
                    int64_t cap = 0, int walk_warps = 4, bool count_only = false);

// Device helper: the distinct neighbor-cell coordinates along one axis (<= 3).
__device__ __forceinline__ int stencil_axis(int c, int nc, bool per, int* out) {
  int cnt = 0;
  for (int d = -1; d <= 1; d++) {
    int k = c + d;  // c is in 0..nc-1, so one wrap suffices
    if (per) {
      k = k < 0 ? k + nc : (k >= nc ? k - nc : k);
    } else if (k < 0 || k >= nc) {
      continue;
    }
    bool dup = false;
    for (int q = 0; q < cnt; q++) dup |= (out[q] == k);
    if (!dup) out[cnt++] = k;
  }
  return cnt;
}
// The 27-cell stencil of cell c as contiguous ranges of the cell-sorted slot array:
// x-adjacent cells of one (z, y) row are consecutive unless the row wraps, so there are
// at most 9 rows of at most 3 ranges (usually 9 ranges in all).
struct StencilRanges {
  int n;
  int32_t beg[27], end[27];  // slots (every entry point keeps n below 2^31)
};
__device__ __forceinline__ void stencil_ranges(const ConfGrid& g, const int* c, const int64_t* __restrict__ cell_start,
                                               StencilRanges& R) {
  int sx[3], sy[3], sz[3];
  const int nx = stencil_axis(c[0], g.nc[0], !isinf(g.L[0]), sx);
  const int ny = stencil_axis(c[1], g.nc[1], !isinf(g.L[1]), sy);
  const int nz = stencil_axis(c[2], g.nc[2], !isinf(g.L[2]), sz);
  // x cells ascending, then runs of consecutive cells merge into one range
  for (int a = 1; a < nx; a++)
    for (int b = a; b > 0 && sx[b - 1] > sx[b]; b--) {
      int t = sx[b];
      sx[b] = sx[b - 1];
      sx[b - 1] = t;
    }
  R.n = 0;
  for (int a = 0; a < nz; a++)
    for (int b = 0; b < ny; b++) {
      const int64_t row = g.cell_off + ((int64_t)sz[a] * g.nc[1] + sy[b]) * g.nc[0];
      int d = 0;
      while (d < nx) {
        int e = d;
        while (e + 1 < nx && sx[e + 1] == sx[e] + 1) e++;
        R.beg[R.n] = (int32_t)cell_start[row + sx[d]];
        R.end[R.n] = (int32_t)cell_start[row + sx[e] + 1];
        R.n++;
        d = e + 1;
      }
    }
}

__device__ __forceinline__ void cell_coords(const ConfGrid& g, double x, double y, double z, int* c) {
  double p[3] = {x, y, z};
#pragma unroll
  for (int a = 0; a < 3; a++) {
    double w = isinf(g.L[a]) ? p[a] - g.lo[a] : p[a] - g.L[a] * floor(p[a] / g.L[a]);
    int k = (int)floor(w / g.cs[a]);
    k = k < 0 ? 0 : k;
    k = k > g.nc[a] - 1 ? g.nc[a] - 1 : k;
    c[a] = k;
  }
}

// ----------------------------------------------------------------------------------
// Small device reductions.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
