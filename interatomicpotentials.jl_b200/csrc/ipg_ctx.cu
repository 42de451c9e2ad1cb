// ipg_ctx.cu — context lifetime, error reporting, device scratch, status word, scan.
#include <algorithm>
#include <cstdarg>
#include <cstdlib>
#include <condition_variable>
#include <mutex>
#include <thread>

#include <unistd.h>

#include "ipg_internal.cuh"

int ipg_fail(ipg_ctx* ctx, int code, const char* fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    ctx->err = buf;
  }
  return code;
}

int ipg_cuda_check(ipg_ctx* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return IPG_OK;
  // clear the runtime's last-error state, so that a failed call (a launch configuration or an
  // attribute the device refuses) is not reported again by the next launch's check
  cudaGetLastError();
  if (e == cudaErrorMemoryAllocation) return ipg_fail(ctx, IPG_ERR_NOMEM, "%s: %s", what, cudaGetErrorString(e));
  return ipg_fail(ctx, IPG_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int ipg_scratch(ipg_ctx* ctx, const char* name, size_t bytes, void** out) {
  DevBuf& b = ctx->bufs[name];
  if (b.cap < bytes) {
    if (ctx->capturing)
      return ipg_fail(ctx, IPG_ERR_CAPACITY, "scratch '%s' would grow during graph capture", name);
    ctx->scratch_gen++;
    if (b.p) {
      // The stream may still use the old buffer.
      CUDA_RET(ctx, cudaStreamSynchronize(ctx->stream));
      CUDA_RET(ctx, cudaFree(b.p));
      b.p = nullptr;
      b.cap = 0;
    }
    size_t cap = bytes + bytes / 8 + 256;
    cudaError_t e = cudaMalloc(&b.p, cap);
    if (e != cudaSuccess) {
      b.p = nullptr;
      cudaGetLastError();
      return ipg_fail(ctx, IPG_ERR_NOMEM, "device allocation of %zu bytes for '%s' failed", cap, name);
    }
    b.cap = cap;
  }
  *out = b.p;
  return IPG_OK;
}

int ipg_status_reset(ipg_ctx* ctx) {
  CUDA_RET(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
  return IPG_OK;
}

int ipg_sync(ipg_ctx* ctx) {
  CUDA_RET(ctx, cudaStreamSynchronize(ctx->stream));
  return IPG_OK;
}

int ipg_side_begin(ipg_ctx* ctx) {
  IPG_RET(ipg_side_join(ctx));
  if (!ctx->side_enabled) return IPG_OK;
  if (!ctx->side) {
    CUDA_RET(ctx, cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
    CUDA_RET(ctx, cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
    CUDA_RET(ctx, cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming));
  }
  CUDA_RET(ctx, cudaEventRecord(ctx->ev_fork, ctx->stream));
  CUDA_RET(ctx, cudaStreamWaitEvent(ctx->side, ctx->ev_fork, 0));
  ctx->side_main = ctx->stream;
  ctx->stream = ctx->side;
  return IPG_OK;
}

int ipg_side_end(ipg_ctx* ctx) {
  if (!ctx->side_main) return IPG_OK;
  ctx->stream = ctx->side_main;
  ctx->side_main = nullptr;
  CUDA_RET(ctx, cudaEventRecord(ctx->ev_join, ctx->side));
  ctx->side_pending = true;
  return IPG_OK;
}

int ipg_side_join(ipg_ctx* ctx) {
  if (ctx->side_main) IPG_RET(ipg_side_end(ctx));  // an error path left the side stream current
  if (!ctx->side_pending) return IPG_OK;
  ctx->side_pending = false;
  CUDA_RET(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0));
  return IPG_OK;
}

int ipg_status_check(ipg_ctx* ctx, const char* what) {
  IPG_RET(ipg_side_join(ctx));
  CUDA_RET(ctx, cudaMemcpyAsync(ctx->h_status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_RET(ctx, cudaStreamSynchronize(ctx->stream));
  int st = *ctx->h_status;
  if (st == IPG_ERR_CAPACITY) return ipg_fail(ctx, st, "%s: device capacity exceeded", what);
  if (st == IPG_ERR_NONFINITE) return ipg_fail(ctx, st, "%s: non-finite position", what);
  if (st == IPG_ERR_SPECIES) return ipg_fail(ctx, st, "%s: species id out of range", what);
  if (st != IPG_OK) return ipg_fail(ctx, st, "%s: device status %d", what, st);
  return IPG_OK;
}

// ---------------------------------------------------------------------------------
// Pinned staging of large host copies.

// A fixed team of host threads that splits one large memcpy: the caller copies the first
// share, each worker one of the others.  Created at a context's first large copy, joined when
// the context is destroyed.  A process forked after the team started has no workers, so the
// team copies on the caller's thread alone there.
struct HostCopyTeam {
  explicit HostCopyTeam(int nthreads) : pid_(getpid()), parts_(nthreads) {
    for (int k = 1; k < nthreads; k++) th_.emplace_back([this, k] { work(k); });
  }
  ~HostCopyTeam() {
    {
      std::lock_guard<std::mutex> lk(m_);
      stop_ = true;
    }
    go_.notify_all();
    for (auto& t : th_) t.join();
  }
  void copy(void* dst, const void* src, size_t bytes) {
    if (th_.empty() || bytes < (size_t(1) << 20) || getpid() != pid_) {
      memcpy(dst, src, bytes);
      return;
    }
    {
      std::lock_guard<std::mutex> lk(m_);
      dst_ = static_cast<char*>(dst);
      src_ = static_cast<const char*>(src);
      bytes_ = bytes;
      left_ = (int)th_.size();
      gen_++;
    }
    go_.notify_all();
    part(0);
    std::unique_lock<std::mutex> lk(m_);
    done_.wait(lk, [this] { return left_ == 0; });
  }

 private:
  // share k of the current copy (shares are whole multiples of 4 KiB; the last takes the rest)
  void part(int k) {
    const size_t share = ((bytes_ / parts_) + 4095) & ~size_t(4095);
    const size_t lo = std::min(bytes_, share * k), hi = k == parts_ - 1 ? bytes_ : std::min(bytes_, lo + share);
    if (hi > lo) memcpy(dst_ + lo, src_ + lo, hi - lo);
  }
  void work(int k) {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(m_);
        go_.wait(lk, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
      }
      part(k);
      std::lock_guard<std::mutex> lk(m_);
      if (--left_ == 0) done_.notify_one();
    }
  }
  const pid_t pid_;
  const int parts_;
  std::vector<std::thread> th_;
  std::mutex m_;
  std::condition_variable go_, done_;
  char* dst_ = nullptr;
  const char* src_ = nullptr;
  size_t bytes_ = 0;
  uint64_t gen_ = 0;
  int left_ = 0;
  bool stop_ = false;
};

namespace {
constexpr size_t PIN_CHUNK = size_t(4) << 20;   // bytes per ring slot
constexpr size_t PIN_DIRECT = size_t(1) << 20;  // smaller copies go straight through the driver
constexpr int SLOTS = ipg_ctx::PIN_SLOTS;

// True when p is page-locked host memory that the device can copy from directly.
bool host_is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

int pinned_ring(ipg_ctx* ctx) {
  for (int k = 0; k < SLOTS; k++) {
    if (!ctx->pinned[k]) {
      void* p = nullptr;
      if (cudaMallocHost(&p, PIN_CHUNK) != cudaSuccess) {
        cudaGetLastError();
        return ipg_fail(ctx, IPG_ERR_NOMEM, "pinned staging allocation failed");
      }
      ctx->pinned[k] = static_cast<char*>(p);
    }
    if (!ctx->pinned_ev[k]) CUDA_RET(ctx, cudaEventCreateWithFlags(&ctx->pinned_ev[k], cudaEventDisableTiming));
  }
  if (!ctx->copy_team) {
    int nt = ctx->copy_threads;
    if (nt <= 0) {  // half the host's hardware threads, at most 8: a memcpy saturates well before
      const unsigned hw = std::thread::hardware_concurrency();
      nt = (int)std::max(1u, std::min(8u, hw / 2));
    }
    ctx->copy_team = new HostCopyTeam(nt);
  }
  return IPG_OK;
}
}  // namespace

void ipg_copy_team_free(ipg_ctx* ctx) {
  delete ctx->copy_team;
  ctx->copy_team = nullptr;
}

int ipg_copy_d2h(ipg_ctx* ctx, void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return IPG_OK;
  if (bytes < PIN_DIRECT || ctx->capturing || host_is_pinned(dst)) {
    CUDA_RET(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_RET(ctx, cudaStreamSynchronize(ctx->stream));
    return IPG_OK;
  }
  IPG_RET(pinned_ring(ctx));
  const size_t nchunk = (bytes + PIN_CHUNK - 1) / PIN_CHUNK;
  auto issue = [&](size_t c) -> int {
    const size_t off = c * PIN_CHUNK, len = std::min(PIN_CHUNK, bytes - off);
    CUDA_RET(ctx, cudaMemcpyAsync(ctx->pinned[c % SLOTS], static_cast<const char*>(src) + off, len,
                                  cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_RET(ctx, cudaEventRecord(ctx->pinned_ev[c % SLOTS], ctx->stream));
    return IPG_OK;
  };
  for (size_t c = 0; c < nchunk && c < (size_t)SLOTS; c++) IPG_RET(issue(c));
  for (size_t c = 0; c < nchunk; c++) {
    CUDA_RET(ctx, cudaEventSynchronize(ctx->pinned_ev[c % SLOTS]));
    const size_t off = c * PIN_CHUNK, len = std::min(PIN_CHUNK, bytes - off);
    ctx->copy_team->copy(static_cast<char*>(dst) + off, ctx->pinned[c % SLOTS], len);
    if (c + SLOTS < nchunk) IPG_RET(issue(c + SLOTS));
  }
  return IPG_OK;
}

int ipg_copy_h2d(ipg_ctx* ctx, void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return IPG_OK;
  if (bytes < PIN_DIRECT || ctx->capturing || host_is_pinned(src)) {
    CUDA_RET(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return IPG_OK;
  }
  IPG_RET(pinned_ring(ctx));
  const size_t nchunk = (bytes + PIN_CHUNK - 1) / PIN_CHUNK;
  for (size_t c = 0; c < nchunk; c++) {
    if (c >= (size_t)SLOTS) CUDA_RET(ctx, cudaEventSynchronize(ctx->pinned_ev[c % SLOTS]));  // slot's DMA done
    const size_t off = c * PIN_CHUNK, len = std::min(PIN_CHUNK, bytes - off);
    ctx->copy_team->copy(ctx->pinned[c % SLOTS], static_cast<const char*>(src) + off, len);
    CUDA_RET(ctx, cudaMemcpyAsync(static_cast<char*>(dst) + off, ctx->pinned[c % SLOTS], len,
                                  cudaMemcpyHostToDevice, ctx->stream));
    CUDA_RET(ctx, cudaEventRecord(ctx->pinned_ev[c % SLOTS], ctx->stream));
  }
  // the ring is reused by the next copy: wait until the DMAs out of it are done
  for (int k = 0; k < SLOTS && k < (int)nchunk; k++) CUDA_RET(ctx, cudaEventSynchronize(ctx->pinned_ev[k]));
  return IPG_OK;
}

// ---------------------------------------------------------------------------------
// Kernel timing: event pairs per kernel name, resolved when read.
int ipg_timing_mark(ipg_ctx* ctx, const char* name, bool start) {
  if (!ctx->timing) return IPG_OK;
  cudaEvent_t e;
  if (!ctx->event_pool.empty()) {
    e = ctx->event_pool.back();
    ctx->event_pool.pop_back();
  } else {
    CUDA_RET(ctx, cudaEventCreate(&e));
  }
  CUDA_RET(ctx, cudaEventRecord(e, ctx->stream));
  auto& t = ctx->timed[name];
  t.ev.push_back(e);
  if (!start) t.launches++;
  return IPG_OK;
}

static int timing_resolve(ipg_ctx* ctx) {
  for (auto& kv : ctx->timed) {
    auto& t = kv.second;
    for (size_t q = 0; q + 1 < t.ev.size(); q += 2) {
      CUDA_RET(ctx, cudaEventSynchronize(t.ev[q + 1]));
      float ms = 0.f;
      CUDA_RET(ctx, cudaEventElapsedTime(&ms, t.ev[q], t.ev[q + 1]));
      t.ms += ms;
      ctx->event_pool.push_back(t.ev[q]);
      ctx->event_pool.push_back(t.ev[q + 1]);
    }
    t.ev.clear();
  }
  return IPG_OK;
}

// ---------------------------------------------------------------------------------
// Exclusive scan, three phases: per-block scan (2048 items per block), scan of block
// sums (recursive), add block offsets.
namespace {
constexpr int SCAN_T = 512;
constexpr int SCAN_PER = 4;
constexpr int SCAN_BLOCK = SCAN_T * SCAN_PER;

__global__ void k_scan_block(const int64_t* __restrict__ in, int64_t* __restrict__ out, int64_t n,
                             int64_t* __restrict__ bsum) {
  __shared__ int64_t wsum[SCAN_T / 32];
  int64_t base = (int64_t)blockIdx.x * SCAN_BLOCK + (int64_t)threadIdx.x * SCAN_PER;
  int64_t v[SCAN_PER];
  int64_t run = 0;
#pragma unroll
  for (int q = 0; q < SCAN_PER; q++) {
    int64_t idx = base + q;
    int64_t x = idx < n ? in[idx] : 0;
    v[q] = run;
    run += x;
  }
  // inclusive warp scan of per-thread totals
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int64_t incl = run;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int64_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  if (w == 0) {
    int64_t s = lane < SCAN_T / 32 ? wsum[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int64_t t = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += t;
    }
    if (lane < SCAN_T / 32) wsum[lane] = s;
  }
  __syncthreads();
  int64_t excl = incl - run + (w > 0 ? wsum[w - 1] : 0);
#pragma unroll
  for (int q = 0; q < SCAN_PER; q++) {
    int64_t idx = base + q;
    if (idx < n) out[idx] = excl + v[q];
  }
  if (threadIdx.x == SCAN_T - 1) bsum[blockIdx.x] = excl + run;
}

__global__ void k_scan_add(int64_t* __restrict__ out, int64_t n, const int64_t* __restrict__ boff) {
  int64_t idx = (int64_t)blockIdx.x * SCAN_BLOCK + threadIdx.x;
  int64_t add = boff[blockIdx.x];
#pragma unroll
  for (int q = 0; q < SCAN_PER; q++, idx += SCAN_T)
    if (idx < n) out[idx] += add;
}
}  // namespace

static int scan_level(ipg_ctx* ctx, const int64_t* in, int64_t* out, int64_t n, int depth) {
  int64_t nb = (n + SCAN_BLOCK - 1) / SCAN_BLOCK;
  if (nb < 1) nb = 1;
  char name[32];
  snprintf(name, sizeof(name), "scan_bsum%d", depth);
  int64_t* bsum;
  IPG_RET(scratch(ctx, name, (size_t)nb + 1, &bsum));
  IPG_LAUNCH(ctx, k_scan_block, (unsigned)nb, SCAN_T, 0, in, out, n, bsum);
  if (nb > 1) {
    IPG_RET(scan_level(ctx, bsum, bsum, nb, depth + 1));
    IPG_LAUNCH(ctx, k_scan_add, (unsigned)nb, SCAN_T, 0, out, n, bsum);
  }
  return IPG_OK;
}

int ipg_scan_i64(ipg_ctx* ctx, const int64_t* in, int64_t* out, int64_t n_plus_1) {
  if (n_plus_1 <= 0) return IPG_OK;
  return scan_level(ctx, in, out, n_plus_1, 0);
}

// ---------------------------------------------------------------------------------
extern "C" {

int ipg_version(void) { return 100; }

int ipg_create(int device, ipg_ctx** out) {
  if (!out) return IPG_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return IPG_ERR_NODEVICE;
  }
  if (device < 0 || device >= ndev) return IPG_ERR_ARG;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return IPG_ERR_CUDA;
  if (prop.major != 10) return IPG_ERR_NODEVICE;  // built for sm_100a only
  {  // the kernels in this library must be sm_100 code that this device can run
    int dev0 = 0;
    cudaGetDevice(&dev0);
    cudaFuncAttributes fa;
    const bool ok = cudaSetDevice(device) == cudaSuccess &&
                    cudaFuncGetAttributes(&fa, k_scan_add) == cudaSuccess && fa.binaryVersion == 100;
    cudaGetLastError();
    cudaSetDevice(dev0);
    if (!ok) return IPG_ERR_NODEVICE;
  }
  ipg_ctx* ctx = new ipg_ctx();
  ctx->device = device;
  ctx->num_sms = prop.multiProcessorCount;
  if (const char* e = getenv("IPG_WALK_BY_ATOM")) ctx->walk_by_cell = e[0] != '1';
  if (const char* e = getenv("IPG_PAIR_FULL")) ctx->pair_full_stencil = e[0] == '1';
  if (const char* e = getenv("IPG_PAIR_MINB")) ctx->pair_minb = std::max(3, std::min(5, atoi(e)));
  if (const char* e = getenv("IPG_WALK_SINGLE")) ctx->walk_single = e[0] != '0';
  if (const char* e = getenv("IPG_SIDE_STREAM")) ctx->side_enabled = e[0] != '0';
  if (const char* e = getenv("IPG_COPY_THREADS")) ctx->copy_threads = std::max(1, std::min(64, atoi(e)));
  int dev0 = 0;
  cudaGetDevice(&dev0);
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&ctx->d_status, sizeof(int)) != cudaSuccess ||
      cudaMallocHost(&ctx->h_status, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    delete ctx;
    return IPG_ERR_CUDA;
  }
  ctx->stream = ctx->own_stream;
  cudaMemset(ctx->d_status, 0, sizeof(int));
  cudaDeviceSynchronize();
  *out = ctx;
  return IPG_OK;
}

int ipg_destroy(ipg_ctx* ctx) {
  if (!ctx) return IPG_ERR_ARG;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->side) cudaStreamSynchronize(ctx->side);
  for (auto& kv : ctx->bufs)
    if (kv.second.p) cudaFree(kv.second.p);
  for (auto& kv : ctx->timed)
    for (cudaEvent_t e : kv.second.ev) cudaEventDestroy(e);
  for (cudaEvent_t e : ctx->event_pool) cudaEventDestroy(e);
  if (ctx->d_status) cudaFree(ctx->d_status);
  if (ctx->h_status) cudaFreeHost(ctx->h_status);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  if (ctx->side) cudaStreamDestroy(ctx->side);
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
  ipg_copy_team_free(ctx);
  for (auto& g : ctx->pair_graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  for (int k = 0; k < ipg_ctx::PIN_SLOTS; k++) {
    if (ctx->pinned[k]) cudaFreeHost(ctx->pinned[k]);
    if (ctx->pinned_ev[k]) cudaEventDestroy(ctx->pinned_ev[k]);
  }
  delete ctx;
  return IPG_OK;
}

const char* ipg_last_error(const ipg_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int ipg_set_stream(ipg_ctx* ctx, void* stream) {
  if (!ctx) return IPG_ERR_ARG;
  ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
  return IPG_OK;
}

int ipg_timing_enable(ipg_ctx* ctx, int on) {
  if (!ctx) return IPG_ERR_ARG;
  if (!on) IPG_RET(timing_resolve(ctx));
  ctx->timing = on != 0;
  return IPG_OK;
}

int ipg_timing_read(ipg_ctx* ctx, const char* kernel, double* total_ms, int64_t* launches) {
  if (!ctx || !kernel) return IPG_ERR_ARG;
  IPG_RET(timing_resolve(ctx));
  auto it = ctx->timed.find(kernel);
  if (total_ms) *total_ms = it == ctx->timed.end() ? 0.0 : it->second.ms;
  if (launches) *launches = it == ctx->timed.end() ? 0 : it->second.launches;
  if (it != ctx->timed.end()) {
    it->second.ms = 0.0;
    it->second.launches = 0;
  }
  return IPG_OK;
}

int ipg_launch_count(const ipg_ctx* ctx, int64_t* out) {
  if (!ctx || !out) return IPG_ERR_ARG;
  *out = ctx->launches;
  return IPG_OK;
}

}  // extern "C"
