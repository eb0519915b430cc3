// Internal declarations shared by the host runtime (*.cpp) and the sm_100a
// kernels (*.cu) of libdelta_gpu.so.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "delta_gpu.h"

namespace dgpu {

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------

// Thrown inside the library only; every C entry point catches and converts.
struct Failure : std::runtime_error {
  int code;
  Failure(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void fail(int code, const std::string& msg);
// Last error of the calling thread's context-free entry points (dgpu_last_error(NULL)).
std::string& free_error();
void check_cuda(cudaError_t e, const char* what);
// Host -> device copy on `s`. A pageable source of up to 1 MiB goes in pieces
// of at most 32 KiB: such pieces are not queued behind large transfers of
// other streams in the host-to-device copy engine (a 256 KB piece waits for a
// whole 70 MB layer upload of another frame; a 32 KB one does not).
cudaError_t h2d_async(void* dst, const void* src, size_t bytes, cudaStream_t s);

// Recording of a frame segment into a CUDA graph (the batch driver). While the
// calling thread records, host -> device copies go through a pinned arena that
// lives with the context (so the recorded copy nodes read memory that stays
// valid and holds this frame's values), and workspace growth, autotuning,
// stage timing and stream synchronisation are refused: the recording is then
// dropped and the segment run directly.
struct CaptureArena {
  unsigned char* base = nullptr;
  size_t size = 0;
  size_t used = 0;
  bool overflow = false;
};
CaptureArena*& capture_arena();  // this thread's; non-null while recording
inline bool capturing() { return capture_arena() != nullptr; }
// Every kernel launch of the library goes through DGPU_LAUNCH, which also
// counts it (dgpu_launch_count).
void count_launch();
// Raise a kernel's dynamic shared-memory limit to at least `bytes` on the
// current device; never lowers it, so threads launching the same kernel with
// different sizes cannot undo each other's setting between set and launch.
void ensure_dynamic_smem(const void* func, size_t bytes);
#define DGPU_CUDA(call) ::dgpu::check_cuda((call), #call)
#define DGPU_LAUNCH(what) (::dgpu::count_launch(), ::dgpu::check_cuda(cudaGetLastError(), what))

// ---------------------------------------------------------------------------
// Device status word: kernels with a data-dependent loop bound record here
// (never spin or trap). Bits are cleared at the start of each entry point.
// ---------------------------------------------------------------------------
enum StatusBit : unsigned {
  kStatusLoopLimit = 1u << 0,  // union-find / search loop hit its cap
  kStatusBounds = 1u << 1,     // an index check rejected an access
};

// ---------------------------------------------------------------------------
// Workspace: named, growable device slots, so steady-state calls allocate
// nothing. Slots never shrink; contents are not preserved across growth.
// ---------------------------------------------------------------------------
enum Slot : int {
  kSlotInSci, kSlotInRef, kSlotInVarS, kSlotInVarR, kSlotInMaskS, kSlotInMaskR,
  kSlotOutDiff, kSlotOutVar, kSlotOutMask, kSlotOutScore,
  kSlotLattice, kSlotLatticeF, kSlotCellX, kSlotCellY, kSlotTaps, kSlotPhi, kSlotFullFields,
  kSlotTheta, kSlotKnots, kSlotZ,
  kSlotExactBad, kSlotSamples, kSlotSelect, kSlotPsf,
  kSlotSeedPos, kSlotSeedNeg, kSlotLabels, kSlotLabelsNeg, kSlotRootRank, kSlotBlockCounts,
  kSlotCompStats, kSlotCompOut, kSlotBright, kSlotScratch0, kSlotScratch1, kSlotScratch2,
  kSlotFit0, kSlotFit1, kSlotFit2, kSlotFit3, kSlotFit4, kSlotFit5, kSlotFit6, kSlotFit7,
  kSlotFit8, kSlotFit9, kSlotFit10, kSlotFit11, kSlotFit12, kSlotFit13, kSlotFit14, kSlotFit15,
  kSlotFft0, kSlotFft1, kSlotFft2, kSlotFft3, kSlotFft4, kSlotFft5,
  kSlotGlsPart, kSlotLdlt,
  kSlotGrad0, kSlotGrad1, kSlotGrad2, kSlotGrad3, kSlotGrad4, kSlotGrad5, kSlotGrad6, kSlotGrad7,
  kSlotBatch0, kSlotBatch1, kSlotBatch2, kSlotBatch3, kSlotBatch4, kSlotBatch5, kSlotBatch6, kSlotBatch7,
  kSlotBatch8, kSlotBatch9, kSlotBatch10, kSlotBatch11,
  kSlotCount
};

struct Context {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  unsigned* d_status = nullptr;  // device status word (see StatusBit)
  // Iteration cap of each union-find search / link loop of the CCL (per
  // thread); dgpu_set_label_loop_cap lowers it for fault-handling tests.
  static constexpr int kDefaultLabelLoopCap = 1 << 24;
  int label_loop_cap = kDefaultLabelLoopCap;
  // Redo a reduced-precision fit in FP64 when its refinement shows it too
  // inaccurate (dgpu_set_precision_fallback).
  bool precision_fallback = true;
  void* slot_ptr[kSlotCount] = {};
  size_t slot_size[kSlotCount] = {};
  std::string last_error;
  // Host-visible timing: label -> accumulated seconds (DELTA_TIMING). Stage
  // events are recorded without synchronising and resolved when drained.
  std::vector<std::pair<std::string, double>> timing;
  struct PendingStage {
    std::string label;
    cudaEvent_t e0, e1;
  };
  std::vector<PendingStage> pending;
  bool timing_enabled = false;
  // Catalog results of the last dgpu_build_catalog (host copies).
  std::vector<double> cat_d;    // 12 double columns x n
  std::vector<int32_t> cat_i;   // 3 int32 columns x n
  std::vector<uint8_t> cat_u8;  // 7 uint8 columns x n
  int cat_count = 0;
  int64_t cat_npix = 0;         // label image size of the last catalog

  // Read-backs (read_back / sync_reads): a mapped pinned area that the host
  // logic's small device -> host copies reach by SM stores, and the copies
  // still to be scattered to their destinations at the next sync_reads.
  struct ReadBack {
    void* host;
    const void* dev;  // copied into the area at the next sync_reads
    size_t off, bytes;
  };
  unsigned char* rb_host = nullptr;
  unsigned char* rb_dev = nullptr;  // rb_host's device address
  size_t rb_used = 0;
  std::vector<ReadBack> rb_items;

  // Recorded frame segments of the batch driver: key (shape and layer
  // configuration) -> executable graph (nullptr: seen once, not recorded
  // yet), and the pinned arena their copy nodes read.
  std::map<std::string, cudaGraphExec_t> graphs;
  CaptureArena arena;

  void* slot(Slot s, size_t bytes);
};

// Keep freed blocks in the device's default memory pool (the workspace slots
// grow from it stream-ordered); once per device.
void keep_pool_memory(int device);

// Process-wide autotuner for launch parameters that do not change a kernel's
// results (e.g. a tile height whose per-pixel arithmetic order is fixed): the
// first call with a new key times every candidate on the call's own data (one
// warm launch, then one launch between CUDA events on the stream) and keeps
// the fastest; later calls reuse it. DELTA_AUTOTUNE=0 skips the timing and
// takes the first candidate (the heuristic choice).
class Autotuner {
 public:
  // Cached choice for key, or -1.
  int lookup(const std::string& key);
  void store(const std::string& key, int choice, const std::vector<std::pair<int, float>>& timings);
  bool enabled() const { return enabled_; }
  std::string report();
  Autotuner();

 private:
  std::mutex mu_;
  std::map<std::string, std::pair<int, std::vector<std::pair<int, float>>>> table_;
  bool enabled_ = true;
};
Autotuner& autotuner();

// Pick among `cands` (the first is the heuristic default) for `key`, launching
// launch(candidate) on stream s; every launch must write the same outputs.
template <class Launch>
int autotune(cudaStream_t s, const std::string& key, const std::vector<int>& cands, Launch&& launch) {
  Autotuner& t = autotuner();
  const int cached = t.lookup(key);
  if (cached >= 0) {
    launch(cached);
    return cached;
  }
  if (capturing()) fail(DGPU_ERR_RUNTIME, "autotuning while recording a graph");
  if (!t.enabled() || cands.size() == 1) {
    launch(cands.front());
    t.store(key, cands.front(), {});
    return cands.front();
  }
  cudaEvent_t e0, e1;
  DGPU_CUDA(cudaEventCreate(&e0));
  DGPU_CUDA(cudaEventCreate(&e1));
  std::vector<std::pair<int, float>> times;
  int best = cands.front();
  float best_ms = 0.0f;
  for (int cand : cands) {
    launch(cand);  // warm (first launch of a template, L2 state)
    DGPU_CUDA(cudaEventRecord(e0, s));
    launch(cand);
    DGPU_CUDA(cudaEventRecord(e1, s));
    DGPU_CUDA(cudaEventSynchronize(e1));
    float ms = 0.0f;
    DGPU_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    times.emplace_back(cand, ms);
    if (times.size() == 1 || ms < best_ms) {
      best_ms = ms;
      best = cand;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  t.store(key, best, times);
  return best;
}

// RAII: clear the status word at entry, check it (after a sync) at exit.
void reset_status(Context& c);
void check_status(Context& c);  // synchronises the stream

// Device -> host read-backs of the host logic. read_back(c, host, dev, bytes)
// names `bytes` of device memory to bring back; `host` holds them only after
// the next sync_reads, which copies every named range (as it is once the work
// queued before the sync has run, so no work queued between read_back and
// sync_reads may change a named range), synchronises the stream and scatters
// the bytes (so `host` must stay valid until then). Up to 1 MiB per sync goes
// by SM stores into the context's mapped pinned area, all ranges in one
// launch: every stream's device-to-host copy-engine transfers share one queue
// in submission order, and a read-back queued there behind another frame's
// 200 MB download waits for all of it. Larger reads, and reads while a graph
// is recorded, take that queue at once. Entry points drop read-backs that an
// error left unscattered.
void read_back(Context& c, void* host, const void* dev, size_t bytes);
void sync_reads(Context& c);
void drop_reads(Context& c);

// The body of a context entry point: selects the context's device, drops the
// read-backs an earlier error left unscattered, optionally clears the device
// status word before the body (`reset`) and checks it after (`check`), and maps
// a Failure to its code (anything else to DGPU_ERR_RUNTIME), recording the
// message on the context and as the last context-free error.
template <class F>
int run_entry(dgpu_context* ctx, bool reset, bool check, F&& f) {
  auto* c = reinterpret_cast<Context*>(ctx);
  try {
    if (ctx == nullptr) fail(DGPU_ERR_INVALID, "null context");
    DGPU_CUDA(cudaSetDevice(c->device));
    drop_reads(*c);
    if (reset) reset_status(*c);
    f(*c);
    if (check) check_status(*c);
    return DGPU_OK;
  } catch (const Failure& e) {
    if (c) c->last_error = e.what();
    free_error() = e.what();
    return e.code;
  } catch (const std::exception& e) {
    if (c) c->last_error = e.what();
    free_error() = e.what();
    return DGPU_ERR_RUNTIME;
  }
}
constexpr int kReadBackList = 16;  // ranges per gather launch
struct ReadBackList {
  const unsigned char* src[kReadBackList];
  unsigned char* dst[kReadBackList];
  unsigned long long bytes[kReadBackList];
  int n;
};
void launch_read_back(cudaStream_t s, const ReadBackList& l);

// Resolve the pending stage events into `timing` (synchronises the stream).
void resolve_timing(Context& c);
unsigned long long launch_count();

// Device-side timing scope keyed by a reference DELTA_TIMING label.
struct StageTimer {
  Context& c;
  std::string label;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  StageTimer(Context& ctx, const char* l);
  ~StageTimer();
};

// Copy a caller array into a device slot (mem == HOST) or return it in place.
const void* stage_in(Context& c, int mem, const void* p, size_t bytes, Slot s);
// Destination for an output: device slot (HOST) or the caller pointer (DEVICE).
void* out_buf(Context& c, int mem, void* p, size_t bytes, Slot s);
// Copy a device slot result back to the caller (HOST mode only).
void stage_out(Context& c, int mem, void* host, const void* dev, size_t bytes);

// ---------------------------------------------------------------------------
// Host math: basis (basis.cpp) and thin-plate spline (tps.cpp)
// ---------------------------------------------------------------------------
struct Basis {
  double beta = 0;
  int n_max = 0, radius = 0, ks = 0, nc = 0;
  std::vector<double> b1d;           // (n_max+1) x ks
  std::vector<std::pair<int, int>> orders;  // (nx, ny) per component
  Basis(double beta, int n_max, int radius);  // radius <= 0 -> default
  std::vector<float> taps() const;   // float32 (n_max+1) x ks
  // The 1-D functions sampled at the offsets shifted by d, g_n(u - d), and
  // their derivatives g_n'(u - d) (FP64, (n_max+1) x ks each).
  void shifted_taps(double d, std::vector<double>& g, std::vector<double>& dg) const;
  std::vector<float> kernel2d(int c) const;
  std::vector<double> component_sums() const;
};
int default_radius(double beta, int n_max);

struct ThinPlate {
  int k = 0;
  double cx = 0, cy = 0, scale = 1;
  std::vector<double> kn;       // k x 2 normalised knots
  std::vector<double> z;        // k x (k-3) null space, row-major
  std::vector<double> penalty;  // k x k
  explicit ThinPlate(const double* knots, int k);
  void design_row(double x, double y, double* out) const;  // k values
  double min_knot_spacing() const;
  // F (P x (nc+1)*r, row-major) with F F^T = blockdiag(penalty) (solve.cpp:47-65).
  std::vector<double> pen_half(int nc, int* r_out) const;
};

// Symmetric eigendecomposition (cyclic Jacobi), ascending eigenvalues.
void sym_eig(int n, const double* a, double* w, double* v);

// Coarse field lattice geometry (subtract.cpp:107-316).
struct FieldGeom {
  bool exact = false;
  int stride = 1, ncx = 0, ncy = 0;
  std::vector<int> gx, gy, cellx, celly;
  std::vector<float> wx, wy;
};
FieldGeom make_field_geom(const ThinPlate& tp, int w, int h);

// ---------------------------------------------------------------------------
// Device fields: lattice (coarse) or full-resolution arrays (exact).
// ---------------------------------------------------------------------------
struct DevFields {
  int exact = 0;
  int nf = 0, w = 0, h = 0;
  const float* full = nullptr;   // exact: nf*h*w
  const float* latf = nullptr;   // coarse: nf*ncy*ncx, float32 copies of the FP64 lattice
  const double* lat = nullptr;   // coarse FP64 lattice
  int ncx = 0, ncy = 0;
  int stride = 0;                // coarse: lattice spacing in pixels (cells of `stride`, the last extended)
  const int* cellx = nullptr;    // w
  const float* wx = nullptr;     // w
  const int* celly = nullptr;    // h
  const float* wy = nullptr;     // h
  const int* gx = nullptr;       // coarse: lattice x coordinates (ncx)
  const int* gy = nullptr;       // coarse: lattice y coordinates (ncy)
};

// Evaluate the fields of `theta` (host) on the device.
DevFields build_fields(Context& c, const ThinPlate& tp, const double* theta, int nf, int w, int h);
// Same, with theta already on the device (FP64, nf*k).
DevFields build_fields_dev(Context& c, const ThinPlate& tp, const double* d_theta, int nf, int w,
                           int h);

// ---------------------------------------------------------------------------
// Kernel launchers (defined in the .cu files)
// ---------------------------------------------------------------------------
struct TpsDev {  // thin-plate constants for device evaluation
  const double* kn = nullptr;  // k x 2
  const double* z = nullptr;   // k x (k-3)
  int k = 0;
  double cx = 0, cy = 0, scale = 1;
};
TpsDev upload_tps(Context& c, const ThinPlate& tp);
void launch_lattice(cudaStream_t s, const TpsDev& t, const double* theta, int nf, const int* gx,
                    const int* gy, int ncx, int ncy, double* lat, float* latf);
void launch_exact_fields(cudaStream_t s, const TpsDev& t, const double* theta, int nf, int w, int h,
                         float* full);

struct SubtractArgs {
  int w, h;
  const float* sci;
  const float* ref;
  const uint8_t* ref_mask;
  DevFields F;
  int n_max, ks, nc;
  const float* taps;  // device (n_max+1)*ks
  const int* ord;     // unused placeholder
  const float* fill;  // device scalar (reference fill value)
  float* diff;
};
void launch_model_convolve(cudaStream_t s, const SubtractArgs& a, const Basis& b);
void launch_variance(cudaStream_t s, int w, int h, const DevFields& F, const float* phi, int rk,
                     int nc, const float* var_s, const float* var_r, float* var_out);
void launch_mask(cudaStream_t s, int w, int h, const float* sci, const float* ref,
                 const uint8_t* sm, const uint8_t* rm, double saturation, int r, const float* diff,
                 uint8_t* mask_out, uint8_t* exact_bad);
void launch_mask_fill(cudaStream_t s, int64_t n, const uint8_t* mask, const uint8_t* exact_bad,
                      const float* fill, float* diff, float* var);
void launch_model_convolve_orders(cudaStream_t s, const SubtractArgs& a, const int2* orders, bool stack);
void launch_photometric_scale(cudaStream_t s, const DevFields& F, const float* sums, int nc, float* out);
// Both middle ranks of z^2 = D^2 / Var (FP64) over the good pixels: after the
// call state[3] / state[4] hold the keys (bit patterns) of ranks (m-1)/2 and
// m/2, state[0] = m. keys: n entries; hist: 512 uints.
void launch_z2_median(cudaStream_t s, int64_t n, const float* d, const float* v, const uint8_t* m,
                      unsigned long long* keys, unsigned long long* state, unsigned int* hist);
void launch_scale_fill(cudaStream_t s, int64_t n, float* v, float scale, bool fill, float value);
void launch_negate(cudaStream_t s, int64_t n, float* v);
// Background median / MAD of a device image with a fixed file-scope scratch
// (no allocation); out2 (host) = {median, MAD}. Synchronises `s`.
void background_noalloc(int64_t n, const float* img, const uint8_t* mask, cudaStream_t s, float* out2);

// Upper median (element size/2 of the sorted sample) of values[7j] that pass a
// predicate, via radix select. Result written to a device float.
enum SampleKind { kSampleReference = 0, kSampleDifference = 1 };
void launch_strided_median(Context& c, int kind, int64_t n, const float* values, const uint8_t* mask,
                           float* d_result);

void launch_matched_filter(cudaStream_t s, int w, int h, const float* img, const float* var, const float* psf_dev,
                           int ps, float sumpsf2, float* out, int* nf_buf);

void launch_basis_convolve(cudaStream_t s, int w, int h, const float* img, const Basis& b,
                           const float* taps, float* out);

// Catalog (k_ccl.cu)
struct CatalogDevResult;
int run_catalog(Context& c, int w, int h, const float* score, const float* diff,
                const uint8_t* mask, const dgpu_catalog_params& p, const float* variance,
                const float* psf, int psf_size, const double* bright_x, const double* bright_y,
                int n_bright);

}  // namespace dgpu
