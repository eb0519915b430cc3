// Host runtime of libdelta_gpu.so: errors, context, workspace slots, staging,
// device-event stage timers, device field set-up.
#include <cuda_runtime.h>

#include <atomic>
#include <map>
#include <mutex>
#include <utility>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>

#include <algorithm>

#include "internal.h"

namespace dgpu {


void fail(int code, const std::string& msg) { throw Failure(code, msg); }

void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) fail(DGPU_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

CaptureArena*& capture_arena() {
  static thread_local CaptureArena* a = nullptr;
  return a;
}

cudaError_t h2d_async(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (CaptureArena* a = capture_arena()) {
    const size_t off = (a->used + 15) & ~size_t(15);
    if (off + bytes > a->size) {
      a->used = off + bytes;
      a->overflow = true;
      return cudaErrorMemoryAllocation;
    }
    std::memcpy(a->base + off, src, bytes);
    a->used = off + bytes;
    return cudaMemcpyAsync(dst, a->base + off, bytes, cudaMemcpyHostToDevice, s);
  }
  constexpr size_t kPiece = size_t(32) << 10, kSplitMax = size_t(1) << 20;
  if (bytes <= kPiece || bytes > kSplitMax)
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
  cudaPointerAttributes pa{};
  if (cudaPointerGetAttributes(&pa, src) != cudaSuccess) {
    cudaGetLastError();
    pa.type = cudaMemoryTypeUnregistered;
  }
  if (pa.type != cudaMemoryTypeUnregistered) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
  for (size_t off = 0; off < bytes; off += kPiece) {
    const cudaError_t e = cudaMemcpyAsync(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off,
                                          std::min(kPiece, bytes - off), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Workspace grows stream-ordered from the device's memory pool: the old buffer
// is released after the work already queued on this context's stream (which is
// the only stream that uses it) and the new one is valid for the work queued
// after, so growth neither synchronises the stream nor the device (a plain
// cudaFree waits for every stream of the device). The pool keeps freed blocks
// for reuse (release threshold raised once per device in dgpu_create).
static void flush_reads(Context& c);

void* Context::slot(Slot s, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (slot_size[s] >= bytes) return slot_ptr[s];
  if (capturing()) fail(DGPU_ERR_RUNTIME, "workspace growth while recording a graph");
  if (slot_ptr[s]) {
    flush_reads(*this);  // a named read-back range may lie in the buffer freed here
    DGPU_CUDA(cudaFreeAsync(slot_ptr[s], stream));
    slot_ptr[s] = nullptr;
    slot_size[s] = 0;
  }
  const size_t want = bytes + bytes / 8 + 256;
  DGPU_CUDA(cudaMallocAsync(&slot_ptr[s], want, stream));
  slot_size[s] = want;
  return slot_ptr[s];
}

Autotuner::Autotuner() {
  const char* v = std::getenv("DELTA_AUTOTUNE");
  enabled_ = !(v != nullptr && std::string(v) == "0");
}

int Autotuner::lookup(const std::string& key) {
  std::lock_guard<std::mutex> lock(mu_);
  const auto it = table_.find(key);
  return it == table_.end() ? -1 : it->second.first;
}

void Autotuner::store(const std::string& key, int choice, const std::vector<std::pair<int, float>>& timings) {
  std::lock_guard<std::mutex> lock(mu_);
  table_.emplace(key, std::make_pair(choice, timings));  // the first result for a key stays
}

std::string Autotuner::report() {
  std::lock_guard<std::mutex> lock(mu_);
  std::string out;
  for (const auto& [key, v] : table_) {
    out += key + " -> " + std::to_string(v.first);
    if (!v.second.empty()) {
      out += " (";
      for (size_t i = 0; i < v.second.size(); ++i) {
        char buf[64];
        std::snprintf(buf, sizeof(buf), "%s%d: %.4f ms", i ? ", " : "", v.second[i].first, v.second[i].second);
        out += buf;
      }
      out += ")";
    }
    out += "\n";
  }
  return out;
}

Autotuner& autotuner() {
  static Autotuner t;
  return t;
}

void keep_pool_memory(int device) {
  static std::mutex mu;
  static std::map<int, bool> done;
  std::lock_guard<std::mutex> lock(mu);
  if (done[device]) return;
  cudaMemPool_t pool = nullptr;
  DGPU_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
  uint64_t keep = ~uint64_t(0);
  DGPU_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  done[device] = true;
}

void reset_status(Context& c) { DGPU_CUDA(cudaMemsetAsync(c.d_status, 0, sizeof(unsigned), c.stream)); }

void check_status(Context& c) {
  if (capturing()) fail(DGPU_ERR_RUNTIME, "a synchronising check while recording a graph");
  unsigned st = 0;
  read_back(c, &st, c.d_status, sizeof(unsigned));
  sync_reads(c);
  if (st & kStatusLoopLimit) fail(DGPU_ERR_LIMIT, "a device loop hit its iteration cap");
  if (st & kStatusBounds) fail(DGPU_ERR_LIMIT, "a device bounds check rejected an access");
}

constexpr size_t kReadBackBytes = size_t(1) << 20;

void read_back(Context& c, void* host, const void* dev, size_t bytes) {
  if (bytes == 0) return;
  if (!capturing() && c.rb_host == nullptr) {
    void* p = nullptr;
    DGPU_CUDA(cudaHostAlloc(&p, kReadBackBytes, cudaHostAllocMapped));
    void* d = nullptr;
    if (cudaHostGetDevicePointer(&d, p, 0) != cudaSuccess || d == nullptr) {
      cudaFreeHost(p);
      fail(DGPU_ERR_CUDA, "read-back area: no device address for mapped pinned memory");
    }
    c.rb_host = static_cast<unsigned char*>(p);
    c.rb_dev = static_cast<unsigned char*>(d);
    c.rb_used = 0;
  }
  const size_t off = (c.rb_used + 15) & ~size_t(15);
  if (capturing() || off + bytes > kReadBackBytes) {
    DGPU_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, c.stream));
    return;
  }
  c.rb_items.push_back({host, dev, off, bytes});
  c.rb_used = off + bytes;
}

// Queue the copies of the named ranges not yet copied (one launch per 16).
static void flush_reads(Context& c) {
  ReadBackList l{};
  for (auto& it : c.rb_items) {
    if (!it.dev) continue;
    l.src[l.n] = static_cast<const unsigned char*>(it.dev);
    l.dst[l.n] = c.rb_dev + it.off;
    l.bytes[l.n] = it.bytes;
    it.dev = nullptr;
    if (++l.n == kReadBackList) {
      launch_read_back(c.stream, l);
      l.n = 0;
    }
  }
  if (l.n) launch_read_back(c.stream, l);
}

void sync_reads(Context& c) {
  flush_reads(c);
  DGPU_CUDA(cudaStreamSynchronize(c.stream));
  for (const auto& it : c.rb_items) std::memcpy(it.host, c.rb_host + it.off, it.bytes);
  c.rb_items.clear();
  c.rb_used = 0;
}

void drop_reads(Context& c) {
  c.rb_items.clear();
  c.rb_used = 0;
}

static std::mutex g_smem_mu;
static std::map<std::pair<int, const void*>, size_t> g_smem_set;

void ensure_dynamic_smem(const void* func, size_t bytes) {
  int dev = 0;
  DGPU_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_smem_mu);
  size_t& cur = g_smem_set[{dev, func}];
  if (bytes <= cur) return;
  DGPU_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
  cur = bytes;
}

static std::atomic<unsigned long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
unsigned long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

StageTimer::StageTimer(Context& ctx, const char* l) : c(ctx), label(l) {
  if (!c.timing_enabled || capturing()) return;  // recorded segments are not stage-timed
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, c.stream);
}

StageTimer::~StageTimer() {
  if (!c.timing_enabled || !e0) return;
  cudaEventRecord(e1, c.stream);
  c.pending.push_back({label, e0, e1});
}

void resolve_timing(Context& c) {
  if (c.pending.empty()) return;
  cudaStreamSynchronize(c.stream);
  for (auto& p : c.pending) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, p.e0, p.e1);
    cudaEventDestroy(p.e0);
    cudaEventDestroy(p.e1);
    bool found = false;
    for (auto& kv : c.timing)
      if (kv.first == p.label) {
        kv.second += ms * 1e-3;
        found = true;
        break;
      }
    if (!found) c.timing.emplace_back(p.label, ms * 1e-3);
  }
  c.pending.clear();
}

const void* stage_in(Context& c, int mem, const void* p, size_t bytes, Slot s) {
  if (p == nullptr) return nullptr;
  if (mem == DGPU_MEM_DEVICE) return p;
  void* d = c.slot(s, bytes);
  DGPU_CUDA(h2d_async(d, p, bytes, c.stream));
  return d;
}

void* out_buf(Context& c, int mem, void* p, size_t bytes, Slot s) {
  if (mem == DGPU_MEM_DEVICE) {
    if (p == nullptr) fail(DGPU_ERR_INVALID, "missing output buffer");
    return p;
  }
  return c.slot(s, bytes);
}

void stage_out(Context& c, int mem, void* host, const void* dev, size_t bytes) {
  if (mem == DGPU_MEM_DEVICE || host == nullptr) return;
  DGPU_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, c.stream));
}

TpsDev upload_tps(Context& c, const ThinPlate& tp) {
  const int k = tp.k, nr = k - 3;
  std::vector<double> buf(2 * static_cast<size_t>(k) + static_cast<size_t>(k) * std::max(nr, 0));
  std::copy(tp.kn.begin(), tp.kn.end(), buf.begin());
  std::copy(tp.z.begin(), tp.z.end(), buf.begin() + 2 * k);
  double* d = static_cast<double*>(c.slot(kSlotZ, sizeof(double) * buf.size()));
  DGPU_CUDA(h2d_async(d, buf.data(), sizeof(double) * buf.size(), c.stream));
  TpsDev t;
  t.kn = d;
  t.z = d + 2 * k;
  t.k = k;
  t.cx = tp.cx;
  t.cy = tp.cy;
  t.scale = tp.scale;
  return t;
}

DevFields build_fields_dev(Context& c, const ThinPlate& tp, const double* d_theta, int nf, int w, int h) {
  if (tp.k > 64) fail(DGPU_ERR_INVALID, "at most 64 knots are supported");
  if (nf > 64) fail(DGPU_ERR_INVALID, "at most 63 kernel components are supported");
  const FieldGeom g = make_field_geom(tp, w, h);
  const TpsDev t = upload_tps(c, tp);
  DevFields F;
  F.nf = nf;
  F.w = w;
  F.h = h;
  if (g.exact) {
    F.exact = 1;
    float* full = static_cast<float*>(c.slot(kSlotFullFields, sizeof(float) * static_cast<size_t>(nf) * w * h));
    launch_exact_fields(c.stream, t, d_theta, nf, w, h, full);
    F.full = full;
    return F;
  }
  F.exact = 0;
  F.ncx = g.ncx;
  F.ncy = g.ncy;
  F.stride = g.stride;
  std::vector<int> ib;
  ib.insert(ib.end(), g.gx.begin(), g.gx.end());
  ib.insert(ib.end(), g.gy.begin(), g.gy.end());
  ib.insert(ib.end(), g.cellx.begin(), g.cellx.end());
  ib.insert(ib.end(), g.celly.begin(), g.celly.end());
  std::vector<float> fb;
  fb.insert(fb.end(), g.wx.begin(), g.wx.end());
  fb.insert(fb.end(), g.wy.begin(), g.wy.end());
  int* di = static_cast<int*>(c.slot(kSlotCellX, sizeof(int) * ib.size()));
  float* df = static_cast<float*>(c.slot(kSlotCellY, sizeof(float) * fb.size()));
  DGPU_CUDA(h2d_async(di, ib.data(), sizeof(int) * ib.size(), c.stream));
  DGPU_CUDA(h2d_async(df, fb.data(), sizeof(float) * fb.size(), c.stream));
  const size_t nl = static_cast<size_t>(nf) * g.ncx * g.ncy;
  double* lat = static_cast<double*>(c.slot(kSlotLattice, sizeof(double) * nl));
  float* latf = static_cast<float*>(c.slot(kSlotLatticeF, sizeof(float) * nl));
  launch_lattice(c.stream, t, d_theta, nf, di, di + g.ncx, g.ncx, g.ncy, lat, latf);
  F.lat = lat;
  F.latf = latf;
  F.gx = di;
  F.gy = di + g.ncx;
  F.cellx = di + g.ncx + g.ncy;
  F.celly = di + g.ncx + g.ncy + w;
  F.wx = df;
  F.wy = df + w;
  return F;
}

DevFields build_fields(Context& c, const ThinPlate& tp, const double* theta, int nf, int w, int h) {
  const size_t n = static_cast<size_t>(nf) * tp.k;
  double* d = static_cast<double*>(c.slot(kSlotTheta, sizeof(double) * n));
  DGPU_CUDA(h2d_async(d, theta, sizeof(double) * n, c.stream));
  return build_fields_dev(c, tp, d, nf, w, h);
}

}  // namespace dgpu
