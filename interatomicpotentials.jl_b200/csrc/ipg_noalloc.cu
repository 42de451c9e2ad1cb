// ipg_noalloc.cu — the pair-potential evaluation for callers that cannot allocate.
//
// Some callers cannot call cudaMalloc: an MD engine that forbids device allocation
// inside its time loop (it owns all device memory up front), a host that hands the
// library only a stream and device buffers, or code that must not create a library
// context (creating one allocates its stream and status word).  ipg_pair_eval_noalloc
// serves them: it computes the same energy, forces and virial as ipg_pair_eval_dev, but
// every scratch buffer it needs (the cell grid, the cell list, per-block partial sums)
// lives in the file-scope device array `g_scratch` below, of fixed size, which every GPU
// that loads the library holds until the process exits.
//
// Limits: at most NOALLOC_MAX_ATOMS atoms and NOALLOC_MAX_CELLS cells (the cell grid is
// coarsened to fit), at most IPG_MAX_PAIR_TERMS terms.  Larger inputs are rejected with
// IPG_ERR_CAPACITY before anything is launched.
//
// Every call shares g_scratch and keeps the last call's contents: the counters that must
// start at zero are cleared at the start of each call, on the caller's stream.  Calls
// whose work overlaps on the GPU (different streams, or different host threads on the
// same device) race on g_scratch; the caller must serialise them, e.g. by using one
// stream.  The first call on a device looks up the device address of g_scratch
// (cudaGetSymbolAddress, with that device current) and caches it; that first call
// should come before any stream capture.  Device-side input errors are not reported:
// there is no status word to read without a synchronisation.  A non-finite position is
// placed in cell 0 and gives non-finite results; a species id outside 0..63 is clamped
// into that range.
#include <algorithm>
#include <atomic>
#include <mutex>

#include "ipg_pair.cuh"

namespace {

constexpr int64_t NOALLOC_MAX_ATOMS = 65536;
constexpr int64_t NOALLOC_MAX_CELLS = 65536;
constexpr int NA_T = 128;                  // threads per block of the pair kernel
constexpr int NA_WARPS = NA_T / 32;
constexpr int NA_PAIR_BLOCKS = 1184;       // grid of the pair kernel (8 per SM on 148 SMs)

// Layout of g_scratch (bytes, every part 256-aligned).
struct Layout {
  static constexpr size_t grid = 0;                                            // ConfGrid
  static constexpr size_t ncell = 256;                                         // int64 total cells
  static constexpr size_t count = 512;                                         // int64 [MAX_CELLS+1]
  static constexpr size_t fill = count + 8 * (NOALLOC_MAX_CELLS + 32);         // int64 [MAX_CELLS]
  static constexpr size_t cell_of = fill + 8 * (NOALLOC_MAX_CELLS + 32);       // int32 [MAX_ATOMS]
  static constexpr size_t atoms = cell_of + 4 * NOALLOC_MAX_ATOMS;             // int32 [MAX_ATOMS]
  static constexpr size_t spos = atoms + 4 * NOALLOC_MAX_ATOMS;                // double4 [MAX_ATOMS]
  static constexpr size_t partial = spos + 32 * NOALLOC_MAX_ATOMS;             // double [BLOCKS][7]
  static constexpr size_t total = partial + 8 * 7 * (NA_PAIR_BLOCKS + 32);
};

// The scratch memory of ipg_pair_eval_noalloc (about 4.3 MB).
static __device__ __align__(256) unsigned char g_scratch[Layout::total];

// Grid set-up on the device (one block): box, open-axis extents, cell edge >= rcut_max,
// at most NOALLOC_MAX_CELLS cells; clears the cell counters.
__global__ void k_na_setup(int64_t n, const double* __restrict__ pos, double L0, double L1, double L2, double rc,
                           unsigned char* scratch) {
  ConfGrid* g = reinterpret_cast<ConfGrid*>(scratch + Layout::grid);
  __shared__ double mn[3][32], mx[3][32];
  const double Ls[3] = {L0, L1, L2};
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x)
    for (int a = 0; a < 3; a++) {
      lo[a] = fmin(lo[a], pos[3 * i + a]);
      hi[a] = fmax(hi[a], pos[3 * i + a]);
    }
  for (int a = 0; a < 3; a++)
    for (int o = 16; o > 0; o >>= 1) {
      lo[a] = fmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
      hi[a] = fmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
    }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0)
    for (int a = 0; a < 3; a++) {
      mn[a][w] = lo[a];
      mx[a][w] = hi[a];
    }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double rcx = rc * (1.0 + 1e-9);
    int64_t tot = 1;
    double ext[3];
    for (int a = 0; a < 3; a++) {
      double l = INFINITY, h = -INFINITY;
      for (int q = 0; q < (int)(blockDim.x >> 5); q++) {
        l = fmin(l, mn[a][q]);
        h = fmax(h, mx[a][q]);
      }
      g->L[a] = Ls[a];
      if (isinf(Ls[a])) {
        if (!(h >= l) || !isfinite(h - l)) l = h = 0.0;
        g->lo[a] = l;
        ext[a] = h - l;
      } else {
        g->lo[a] = 0.0;
        ext[a] = Ls[a];
      }
      int nc = 1;
      if (rcx > 0.0 && isfinite(rcx) && ext[a] > 0.0) nc = (int)fmax(1.0, fmin(floor(ext[a] / rcx), 1024.0));
      g->nc[a] = nc;
      tot *= nc;
    }
    const int64_t cap = NOALLOC_MAX_CELLS < 8 * n + 64 ? NOALLOC_MAX_CELLS : 8 * n + 64;
    while (tot > cap) {
      int a = (g->nc[0] >= g->nc[1] && g->nc[0] >= g->nc[2]) ? 0 : (g->nc[1] >= g->nc[2] ? 1 : 2);
      tot /= g->nc[a];
      g->nc[a] = g->nc[a] / 2 > 1 ? g->nc[a] / 2 : 1;
      tot *= g->nc[a];
    }
    for (int a = 0; a < 3; a++) g->cs[a] = ext[a] > 0.0 ? ext[a] / g->nc[a] : 1.0;
    g->cell_off = 0;
    g->atom_off = 0;
    g->natoms = n;
    *reinterpret_cast<int64_t*>(scratch + Layout::ncell) = tot;
  }
  int64_t* count = reinterpret_cast<int64_t*>(scratch + Layout::count);
  int64_t* fill = reinterpret_cast<int64_t*>(scratch + Layout::fill);
  for (int64_t c = threadIdx.x; c <= NOALLOC_MAX_CELLS; c += blockDim.x) {
    count[c] = 0;
    if (c < NOALLOC_MAX_CELLS) fill[c] = 0;
  }
}

__global__ void k_na_count(int64_t n, const double* __restrict__ pos, unsigned char* scratch) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const ConfGrid g = *reinterpret_cast<const ConfGrid*>(scratch + Layout::grid);
  double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
  if (!isfinite(x) || !isfinite(y) || !isfinite(z)) x = y = z = 0.0;
  int c[3];
  cell_coords(g, x, y, z, c);
  const int64_t cell = ((int64_t)c[2] * g.nc[1] + c[1]) * g.nc[0] + c[0];
  reinterpret_cast<int32_t*>(scratch + Layout::cell_of)[i] = (int32_t)cell;
  atomicAdd(reinterpret_cast<unsigned long long*>(scratch + Layout::count) + cell, 1ull);
}

// Exclusive scan of the cell counts in place (one block of 1024 threads).
__global__ void k_na_scan(unsigned char* scratch) {
  int64_t* a = reinterpret_cast<int64_t*>(scratch + Layout::count);
  const int64_t m = *reinterpret_cast<const int64_t*>(scratch + Layout::ncell) + 1;
  __shared__ int64_t tot[1024];
  const int64_t per = (m + 1023) / 1024;
  const int64_t b = threadIdx.x * per, e = b + per < m ? b + per : m;
  int64_t s = 0;
  for (int64_t k = b; k < e; k++) s += a[k];
  tot[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 1; k < 1024; k++) tot[k] += tot[k - 1];
  __syncthreads();
  int64_t run = threadIdx.x ? tot[threadIdx.x - 1] : 0;
  for (int64_t k = b; k < e; k++) {
    const int64_t v = a[k];
    a[k] = run;
    run += v;
  }
}

__global__ void k_na_fill(int64_t n, unsigned char* scratch) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t c = reinterpret_cast<const int32_t*>(scratch + Layout::cell_of)[i];
  const int64_t* start = reinterpret_cast<const int64_t*>(scratch + Layout::count);
  unsigned long long q = atomicAdd(reinterpret_cast<unsigned long long*>(scratch + Layout::fill) + c, 1ull);
  reinterpret_cast<int32_t*>(scratch + Layout::atoms)[start[c] + (int64_t)q] = (int32_t)i;
}

__global__ void k_na_sort(unsigned char* scratch) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= *reinterpret_cast<const int64_t*>(scratch + Layout::ncell)) return;
  const int64_t* start = reinterpret_cast<const int64_t*>(scratch + Layout::count);
  int32_t* at = reinterpret_cast<int32_t*>(scratch + Layout::atoms);
  const int64_t s = start[c], e = start[c + 1];
  for (int64_t x = s + 1; x < e; x++) {
    const int32_t v = at[x];
    int64_t y = x - 1;
    while (y >= s && at[y] > v) {
      at[y + 1] = at[y];
      y--;
    }
    at[y + 1] = v;
  }
}

__global__ void k_na_gather(int64_t n, const double* __restrict__ pos, const int32_t* __restrict__ species,
                            unsigned char* scratch) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int32_t i = reinterpret_cast<const int32_t*>(scratch + Layout::atoms)[s];
  int sp = species[i];
  sp = sp < 0 ? 0 : (sp > 63 ? 63 : sp);
  reinterpret_cast<double4*>(scratch + Layout::spos)[s] =
      make_double4(pos[3 * (int64_t)i], pos[3 * (int64_t)i + 1], pos[3 * (int64_t)i + 2], (double)sp);
}

// Warp per atom over the stencil ranges (grid-stride over atoms): the full-stencil walk of
// ipg_pair.cuh, the same code as the context path's fallback kernel.  Per-block partials of
// E and the virial go to scratch, forces to F.
__global__ void __launch_bounds__(NA_T) k_na_pair(const __grid_constant__ PairTerms T, int64_t n,
                                                  unsigned char* scratch, double* __restrict__ F) {
  __shared__ PairHit hits[NA_WARPS][64];
  __shared__ double red[NA_WARPS][7];
  const ConfGrid g = *reinterpret_cast<const ConfGrid*>(scratch + Layout::grid);
  const int64_t* cell_start = reinterpret_cast<const int64_t*>(scratch + Layout::count);
  const int32_t* cell_atoms = reinterpret_cast<const int32_t*>(scratch + Layout::atoms);
  const double4* spos = reinterpret_cast<const double4*>(scratch + Layout::spos);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int64_t s = (int64_t)blockIdx.x * NA_WARPS + w; s < n; s += (int64_t)gridDim.x * NA_WARPS)
    pair_walk_atom(T, g, cell_start, cell_atoms, spos, s, hits[w], lane, acc, F);
#pragma unroll
  for (int k = 0; k < 7; k++) {
    const double v = warp_sum(acc[k]);
    if (lane == 0) red[w][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < 7) {
    double v = 0.0;
    for (int q = 0; q < NA_WARPS; q++) v += red[q][threadIdx.x];
    reinterpret_cast<double*>(scratch + Layout::partial)[(int64_t)blockIdx.x * 7 + threadIdx.x] = v;
  }
}

__global__ void k_na_reduce(int nblocks, const unsigned char* scratch, double* E, double* W6) {
  __shared__ double sm[7][256];
  const double* part = reinterpret_cast<const double*>(scratch + Layout::partial);
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
    for (int k = 0; k < 7; k++) acc[k] += part[7 * b + k];
  for (int k = 0; k < 7; k++) sm[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o)
      for (int k = 0; k < 7; k++) sm[k][threadIdx.x] += sm[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (E) *E = sm[0][0];
    if (W6)
      for (int k = 0; k < 6; k++) W6[k] = sm[1 + k][0];
  }
}

// Device address of g_scratch, looked up once per device (with that device current) and
// published through an atomic slot; the lookup itself runs under a mutex, so concurrent first
// calls from several host threads are safe.  The address belongs to the device's context at
// the lookup; after cudaDeviceReset it is stale (documented in include/ipg.h).
constexpr int NA_MAX_DEVICES = 64;
std::atomic<unsigned char*> g_scratch_ptr[NA_MAX_DEVICES];
std::mutex g_scratch_mu;

int scratch_address(int dev, unsigned char** out) {
  if (dev < 0 || dev >= NA_MAX_DEVICES) return IPG_ERR_ARG;
  unsigned char* p = g_scratch_ptr[dev].load(std::memory_order_acquire);
  if (!p) {
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    p = g_scratch_ptr[dev].load(std::memory_order_relaxed);
    if (!p) {
      void* a = nullptr;
      if (cudaGetSymbolAddress(&a, g_scratch) != cudaSuccess) {
        cudaGetLastError();
        return IPG_ERR_CUDA;
      }
      p = static_cast<unsigned char*>(a);
      g_scratch_ptr[dev].store(p, std::memory_order_release);
    }
  }
  *out = p;
  return IPG_OK;
}

}  // namespace

extern "C" {

int ipg_pair_eval_noalloc(void* stream, int64_t n, const double* d_pos, const int32_t* d_species, const double L[3],
                          const ipg_pair_term* terms, int32_t nterms, double* d_E, double* d_F, double* d_W6,
                          uint32_t flags) {
  if (n < 0 || !L || (n > 0 && (!d_pos || !d_species)) || (nterms > 0 && !terms)) return IPG_ERR_ARG;
  if (nterms < 0 || nterms > IPG_MAX_PAIR_TERMS) return IPG_ERR_ARG;
  if (n > NOALLOC_MAX_ATOMS) return IPG_ERR_CAPACITY;  // beyond the size of g_scratch
  if (((flags & IPG_WANT_E) && !d_E) || ((flags & IPG_WANT_F) && !d_F && n) || ((flags & IPG_WANT_W) && !d_W6))
    return IPG_ERR_ARG;
  for (int a = 0; a < 3; a++)
    if (!(L[a] > 0.0)) return IPG_ERR_ARG;
  PairTerms T;
  char err[256];
  if (pair_prepare_terms(terms, nterms, T, err, sizeof(err)) != IPG_OK) return IPG_ERR_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return IPG_ERR_NODEVICE;
  unsigned char* sc = nullptr;
  IPG_RET(scratch_address(dev, &sc));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned an = (unsigned)std::max<int64_t>(1, (n + 255) / 256);
  k_na_setup<<<1, 1024, 0, st>>>(n, d_pos, L[0], L[1], L[2], T.rcut_max, sc);
  if (n > 0) {
    k_na_count<<<an, 256, 0, st>>>(n, d_pos, sc);
    k_na_scan<<<1, 1024, 0, st>>>(sc);
    k_na_fill<<<an, 256, 0, st>>>(n, sc);
    k_na_sort<<<(unsigned)((NOALLOC_MAX_CELLS + 255) / 256), 256, 0, st>>>(sc);
    k_na_gather<<<an, 256, 0, st>>>(n, d_pos, d_species, sc);
  }
  const int pb = (int)std::min<int64_t>(NA_PAIR_BLOCKS, std::max<int64_t>(1, (n + NA_WARPS - 1) / NA_WARPS));
  k_na_pair<<<pb, NA_T, 0, st>>>(T, n, sc, (flags & IPG_WANT_F) ? d_F : nullptr);
  k_na_reduce<<<1, 256, 0, st>>>(pb, sc, (flags & IPG_WANT_E) ? d_E : nullptr, (flags & IPG_WANT_W) ? d_W6 : nullptr);
  return cudaGetLastError() == cudaSuccess ? IPG_OK : IPG_ERR_CUDA;
}

}  // extern "C"
