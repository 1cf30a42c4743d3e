// gpu_solver.cu — B200 (sm_100a) Levenberg–Marquardt bundle adjustment.
//
// Hot path (reference paths relative to the openmvg-rs root):
//   K1  k_linearize_tiles .. per-observation projection, robust weight, analytic point / camera
//                            Jacobians (one CTA per tile of whole points) and the per-point 3x3
//                            Gram + FP64 damped inverse
//                            (schur/point.rs:176-448, schur/assembly.rs:893-1040, point_block.rs:78-184)
//   K2  k_block_tiles ...... camera-side deterministic segmented sums over the record tiles: U blocks,
//       k_block_records      g, reduced g, damping diagonal, pose/intrinsic edges, diagonal point
//                            coupling (asm_tiles.cuh)
//       k_pairs ............ explicit Schur blocks S_bb' -= W V^-1 W^T (schur/assembly.rs:999-1038)
//   K3  k_block_rows ....... explicit S by block rows (BSR), banded tiled FP64 Cholesky and solves
//                            (explicit_s.cuh; stands in for faer's sparse LLT)
//       k_mv_tiles ......... matrix-free reduced-camera-system product S x (retained/operator.rs:137-227)
//       block-Jacobi PCG ... sparse/pcg.rs:23-119, retained/mod.rs:682-934, retained/block.rs:148-246
//   K4  k_retract, k_candidate_points: step cap, retraction, back-substitution and candidate rule
//                            (optimizer.rs:376-702, sparse/calibrated/candidate.rs:23-333,
//                            schur/point.rs:537-728, point_geometry.rs:110-130)
// Every reduction runs in a fixed order (fixed grid, fixed shuffle trees, fixed chunk order), so a
// solve is bitwise reproducible run to run.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "gpu_solver.hpp"
#include "fixed_rotation.hpp"

#include <atomic>
#include <thread>

namespace omvgba {

#define CUDA_OK(expr)                                                                                 \
  do {                                                                                                \
    cudaError_t _e = (expr);                                                                          \
    if (_e != cudaSuccess)                                                                            \
      throw SolveFailure{8, std::string("CUDA error: ") + cudaGetErrorString(_e) + " at " #expr};     \
  } while (0)

constexpr int kChunk = 256;     // entities per block chunk
constexpr int kReduceThreads = 256;

// Telemetry of the calling thread: kernels launched and host<->device bytes copied. A solve runs
// on the thread that called it, so the report takes the difference across the call.
struct Telemetry {
  uint64_t launches = 0, h2d = 0, d2h = 0;
};
thread_local Telemetry tl_telemetry;

void telemetry_read(uint64_t* launches, uint64_t* h2d, uint64_t* d2h) {
  *launches = tl_telemetry.launches;
  *h2d = tl_telemetry.h2d;
  *d2h = tl_telemetry.d2h;
}

// Every kernel launch goes through this macro so that the report can state how many ran.
#define OMVGBA_LAUNCH(kernel, grid, block, smem, stream, ...)   \
  do {                                                          \
    kernel<<<grid, block, smem, stream>>>(__VA_ARGS__);         \
    ++tl_telemetry.launches;                                    \
  } while (0)

// A launch that, with pdl set, may overlap the end of the previous kernel on the stream
// (programmatic stream serialization; the kernel orders itself with pdl_wait). A failed launch is
// reported by the next launch check, like the <<<>>> launches.
template <typename... KArgs, typename... Args>
void launch_pdl(bool pdl, void (*kernel)(KArgs...), unsigned grid, unsigned block, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr{};
  attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr.val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = pdl ? 1 : 0;
  (void)cudaLaunchKernelEx(&cfg, kernel, args...);
  ++tl_telemetry.launches;
}

// Pinned staging buffer of the calling thread for small host<->device copies: a copy from or to
// pageable memory goes through the driver's shared staging path, which serializes concurrent solves
// on different threads; a copy through pinned memory does not.
struct PinnedStage {
  void* p = nullptr;
  size_t bytes = 0;
  ~PinnedStage() {
    if (p) cudaFreeHost(p);
  }
  void* get(size_t need) {
    if (need <= bytes) return p;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    const size_t size = std::max<size_t>(need, 64 * 1024);
    if (cudaMallocHost(&p, size) != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      return nullptr;
    }
    bytes = size;
    return p;
  }
};
thread_local PinnedStage tl_pinned;
thread_local PinnedStage tl_poll;  // the PCG loop's status mirrors (read while the next batch runs)
constexpr size_t kStagedCopyMax = 1u << 20;

// Large host->device copies from pageable memory: the source is copied by several host threads into
// one of two pinned chunks while the other chunk's DMA runs (an event per chunk guards its reuse).
// Returns when every chunk has reached the device, as a pageable copy would.
constexpr size_t kPipelinedCopyMin = 32u << 20;
constexpr size_t kPipelineChunk = 16u << 20;
struct PinnedRing {
  void* p[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int device = -1;
  bool ready = false;
  ~PinnedRing() {
    for (int i = 0; i < 2; ++i) {
      if (p[i]) cudaFreeHost(p[i]);
      if (ev[i]) cudaEventDestroy(ev[i]);
    }
  }
  bool ensure() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    if (ready && dev == device) return true;
    for (int i = 0; i < 2; ++i) {  // events belong to a device: rebuild them for this one
      if (ev[i]) cudaEventDestroy(ev[i]);
      ev[i] = nullptr;
      if (!p[i] && cudaMallocHost(&p[i], kPipelineChunk) != cudaSuccess) {
        cudaGetLastError();
        p[i] = nullptr;
        return false;
      }
      if (cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        ev[i] = nullptr;
        return false;
      }
    }
    device = dev;
    ready = true;
    return true;
  }
};
thread_local PinnedRing tl_ring;

inline void parallel_memcpy(void* dst, const void* src, size_t bytes) {
  const size_t nt = std::max<size_t>(1, std::min<size_t>(host_thread_limit(), 8));
  const size_t per = ((bytes + nt - 1) / nt + 63) & ~size_t(63);
  std::vector<std::thread> pool;
  for (size_t i = 1; i < nt && i * per < bytes; ++i)
    pool.emplace_back([=] {
      std::memcpy(static_cast<char*>(dst) + i * per, static_cast<const char*>(src) + i * per,
                  std::min(per, bytes - i * per));
    });
  std::memcpy(dst, src, std::min(per, bytes));
  for (auto& t : pool) t.join();
}

inline cudaError_t upload_pipelined(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (!tl_ring.ensure()) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
  cudaError_t e = cudaSuccess;
  size_t i = 0;
  for (size_t off = 0; off < bytes && e == cudaSuccess; off += kPipelineChunk, ++i) {
    const int b = (int)(i & 1);
    const size_t n = std::min(kPipelineChunk, bytes - off);
    if (i >= 2) e = cudaEventSynchronize(tl_ring.ev[b]);  // this chunk's previous copy has landed
    if (e != cudaSuccess) break;
    parallel_memcpy(tl_ring.p[b], static_cast<const char*>(src) + off, n);
    e = cudaMemcpyAsync(static_cast<char*>(dst) + off, tl_ring.p[b], n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaEventRecord(tl_ring.ev[b], st);
  }
  const cudaError_t w = cudaStreamSynchronize(st);
  return e != cudaSuccess ? e : w;
}

// Host<->device copy on `st`, counted in the telemetry. Copies of at most kStagedCopyMax bytes go
// through the thread's pinned stage and have completed when the call returns (callers read the
// host side right after their next synchronize, so nothing relies on them staying asynchronous).
inline cudaError_t copy_async(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, cudaStream_t st) {
  if (kind == cudaMemcpyHostToDevice) tl_telemetry.h2d += bytes;
  if (kind == cudaMemcpyDeviceToHost) tl_telemetry.d2h += bytes;
  if ((kind == cudaMemcpyHostToDevice || kind == cudaMemcpyDeviceToHost) && bytes > 0 && bytes <= kStagedCopyMax) {
    if (void* stage = tl_pinned.get(bytes)) {
      if (kind == cudaMemcpyHostToDevice) {
        std::memcpy(stage, src, bytes);
        cudaError_t e = cudaMemcpyAsync(dst, stage, bytes, kind, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // the stage is reused by the next copy
        return e;
      }
      cudaError_t e = cudaMemcpyAsync(stage, src, bytes, kind, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e == cudaSuccess) std::memcpy(dst, stage, bytes);
      return e;
    }
  }
  if (kind == cudaMemcpyHostToDevice && bytes >= kPipelinedCopyMin) return upload_pipelined(dst, src, bytes, st);
  return cudaMemcpyAsync(dst, src, bytes, kind, st);
}

// ----------------------------------------------------------------------------------------------
// Context
// ----------------------------------------------------------------------------------------------
struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;
  double* pinned = nullptr;  // scalar readback
  size_t pinned_count = 0;
};

int device_count() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

Context* context_create(int device, std::string* error) {
  Context* c = new Context();
  c->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMallocHost(&c->pinned, sizeof(double) * 64);
  if (e != cudaSuccess) {
    if (error) *error = cudaGetErrorString(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return nullptr;
  }
  c->pinned_count = 64;
  return c;
}

int context_device(const Context* c) { return c->device; }
void* context_stream(const Context* c) { return (void*)c->stream; }

void context_destroy(Context* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->pinned) cudaFreeHost(c->pinned);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

// Device bytes held by the calling thread's live DBufs (a solve's workspace is the growth across its
// set-up).
thread_local uint64_t tl_device_bytes = 0;

// Device buffer owned for one solve (stream-ordered allocation).
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t s = nullptr;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  void alloc(size_t count, cudaStream_t stream) {
    release();
    s = stream;
    n = count;
    if (count) {
      CUDA_OK(cudaMallocAsync((void**)&p, sizeof(T) * count, stream));
      tl_device_bytes += sizeof(T) * count;
    }
  }
  void upload(const T* host, size_t count, cudaStream_t stream) {
    alloc(count, stream);
    if (count) CUDA_OK(copy_async(p, host, sizeof(T) * count, cudaMemcpyHostToDevice, stream));
  }
  void zero() {
    if (n) CUDA_OK(cudaMemsetAsync(p, 0, sizeof(T) * n, s));
  }
  void release() {
    if (p) {
      cudaFreeAsync(p, s);
      tl_device_bytes -= sizeof(T) * n;
    }
    p = nullptr;
    n = 0;
  }
  ~DBuf() { release(); }
};

// Uploads v, or, when v holds fewer than min_count elements, a zero-padded copy of it (device
// tables are never empty); a long enough table goes up from its own storage without a host copy.
template <typename T, typename A>
void upload_padded(DBuf<T>& b, const std::vector<T, A>& v, size_t min_count, cudaStream_t st) {
  if (v.size() >= min_count) {
    b.upload(v.data(), v.size(), st);
    return;
  }
  std::vector<T> padded(v.begin(), v.end());
  padded.resize(min_count, T{});
  b.upload(padded.data(), padded.size(), st);
}

// ----------------------------------------------------------------------------------------------
// Device problem view
// ----------------------------------------------------------------------------------------------
struct Gauge {
  int fixed_cam;
  double baseline, scene;
  double dir[3], b0[3], b1[3];
};

struct DevView {
  int P, ncam, self_cal, pixel_model;
  const uint32_t* pt_off;      // P+1
  const uint32_t* obs_cam;     // N
  const double* obs_px;        // N x 2
  const uint32_t* obs_model;   // N (calibrated)
  const FixedCameraDev* models;
  const uint32_t* cam_group;   // ncam
  const int* pose_off;         // ncam
  const int* pose_dim;         // ncam
  const uint8_t* pose_mask;    // ncam: bit 0 rotation, bit 1 translation (3 when the layout is legacy)
  int angular;                 // angular residuals: obs_bearing holds each observation's unit bearing
  const double* obs_bearing;   // N x 3 (angular only)
  const int* intr_off;         // ng
  const int* intr_dim;         // ng
  const uint8_t* fixed_points; // P
};

struct DevState {
  double* pose;    // ncam x 12: R (9) then t (3)
  double* points;  // P x 3
  double* groups;  // ng x 3 (focal, k1, k2)
};

__device__ __forceinline__ RadialDev make_radial(const double* g) {
  RadialDev c;
  c.focal = g[0];
  c.k1 = g[1];
  c.k2 = g[2];
  double t;
  c.has_turn = first_radial_turn_squared(c.k1, c.k2, &t) ? 1 : 0;
  c.turn = t;
  return c;
}

// Projection of observation o for camera point xc; Ji is filled for self-calibration.
__device__ __forceinline__ bool project_obs(const DevView& v, const double* groups, int o, const double xc[3],
                                            double r[2], double J[2][3], double Ji[2][3]) {
  if (v.angular) return angular_linearize(v.obs_bearing + 3 * (size_t)o, xc, r, J);
  double ox = v.obs_px[2 * o], oy = v.obs_px[2 * o + 1];
  if (v.self_cal) {
    RadialDev c = make_radial(groups + 3 * v.cam_group[v.obs_cam[o]]);
    return radial_linearize(c, xc[0], xc[1], xc[2], ox, oy, r, J, Ji);
  }
  const FixedCameraDev& m = v.models[v.obs_model[o]];
  if (v.pixel_model) return pixel_linearize(m, xc[0], xc[1], xc[2], ox, oy, r, J);
  return m.linearize(xc[0], xc[1], xc[2], ox, oy, r, J);
}

// ----------------------------------------------------------------------------------------------
// Deterministic reductions
// ----------------------------------------------------------------------------------------------
template <int NV>
struct RedVec {
  double v[NV];
};

// Per-point linearization summary reduced over points: sums (cost, sq, point_red) and extrema.
struct PointSummary {
  double cost, sq, point_red, grad_norm, min_rcond;
  double invalid, weak, pad;
};

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  return x;
}
__device__ __forceinline__ double warp_max(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_down_sync(0xffffffffu, x, o));
  return x;
}
__device__ __forceinline__ double warp_min(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = fmin(x, __shfl_down_sync(0xffffffffu, x, o));
  return x;
}

// Reduce an array of PointSummary (one per point) into per-block partials; fixed order.
__global__ void k_reduce_summary(const PointSummary* in, int n, PointSummary* out) {
  __shared__ PointSummary sh[kReduceThreads / 32];
  int tid = threadIdx.x;
  PointSummary acc{0, 0, 0, 0, 1.0, 0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + tid; i < n; i += gridDim.x * blockDim.x) {
    PointSummary s = in[i];
    acc.cost += s.cost;
    acc.sq += s.sq;
    acc.point_red += s.point_red;
    acc.grad_norm = fmax(acc.grad_norm, s.grad_norm);
    acc.min_rcond = fmin(acc.min_rcond, s.min_rcond);
    acc.invalid += s.invalid;
    acc.weak += s.weak;
  }
  acc.cost = warp_sum(acc.cost);
  acc.sq = warp_sum(acc.sq);
  acc.point_red = warp_sum(acc.point_red);
  acc.grad_norm = warp_max(acc.grad_norm);
  acc.min_rcond = warp_min(acc.min_rcond);
  acc.invalid = warp_sum(acc.invalid);
  acc.weak = warp_sum(acc.weak);
  if ((tid & 31) == 0) sh[tid >> 5] = acc;
  __syncthreads();
  if (tid == 0) {
    PointSummary t = sh[0];
    for (int w = 1; w < (int)(blockDim.x / 32); ++w) {
      t.cost += sh[w].cost;
      t.sq += sh[w].sq;
      t.point_red += sh[w].point_red;
      t.grad_norm = fmax(t.grad_norm, sh[w].grad_norm);
      t.min_rcond = fmin(t.min_rcond, sh[w].min_rcond);
      t.invalid += sh[w].invalid;
      t.weak += sh[w].weak;
    }
    out[blockIdx.x] = t;
  }
}

// Sum of NV-component records (e.g. dot products) with a fixed grid: per block partial, then the
// final pass over partials in index order.
template <int NV>
__global__ void k_reduce_vec(const RedVec<NV>* in, int n, RedVec<NV>* out) {
  __shared__ double sh[kReduceThreads / 32][NV];
  int tid = threadIdx.x;
  double acc[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) acc[k] = 0.0;
  for (int i = blockIdx.x * blockDim.x + tid; i < n; i += gridDim.x * blockDim.x)
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] += in[i].v[k];
#pragma unroll
  for (int k = 0; k < NV; ++k) acc[k] = warp_sum(acc[k]);
  if ((tid & 31) == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) sh[tid >> 5][k] = acc[k];
  __syncthreads();
  if (tid == 0) {
    RedVec<NV> t;
    for (int k = 0; k < NV; ++k) {
      double s = 0.0;
      for (int w = 0; w < (int)(blockDim.x / 32); ++w) s += sh[w][k];
      t.v[k] = s;
    }
    out[blockIdx.x] = t;
  }
}

// Dot products of D-vectors: out[k] = sum_i a_k[i] * b_k[i], fixed order.
struct DotArgs {
  const double* a[4];
  const double* b[4];
  int count;
};
__global__ void k_dots(DotArgs args, int n, double* out) {
  // single block of 1024 threads: strided partials, fixed shuffle tree, fixed warp order
  __shared__ double sh[32][4];
  int tid = threadIdx.x;
  double acc[4] = {0, 0, 0, 0};
  for (int i = tid; i < n; i += blockDim.x)
    for (int k = 0; k < args.count; ++k) acc[k] += args.a[k][i] * args.b[k][i];
  for (int k = 0; k < 4; ++k) acc[k] = warp_sum(acc[k]);
  if ((tid & 31) == 0)
    for (int k = 0; k < 4; ++k) sh[tid >> 5][k] = acc[k];
  __syncthreads();
  if (tid < args.count) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) s += sh[w][tid];
    out[tid] = s;
  }
}

// ----------------------------------------------------------------------------------------------
// K1: per-point linearization (+ point-block factorization)
// ----------------------------------------------------------------------------------------------
// Per-observation Jacobian record (sqrt-weighted): 2 x 9 camera columns (pose | intrinsics), then
// 2 x 3 point columns: kRec = 24 components. Records are stored tile-blocked and component-major:
// component k of the observation at tile-local index i lives at tile_base + k * rs + i, rs being
// the tile capacity. A tile's block is contiguous and 16 B aligned (one bulk async copy), and
// threads reading one component of consecutive observations hit consecutive shared-memory banks.
constexpr int kRec = 24;
constexpr int kJp = 18;

template <typename T>
struct LinOut {
  T* rec;                  // ntiles x rs x kRec
  const uint32_t* obs_rec; // N: element index of each observation's component 0
  int rs;                  // component stride (tile capacity)
  float* rec32;            // optional FP32 copy of the records for mixed-precision products
  const uint32_t* obs_rec32;
  int rs32;
  double* rw;      // N x 2, sqrt-weighted residual
  double* vinv;    // P x 6: damped point-block inverse (zero for fixed points)
  double* vfac;    // P x 6: its factor N, Vhat^-1 = N^T N (zero for fixed points), for the tile product
  double* ig;      // P x 3: Vhat^-1 g_p (zero for fixed points)
  double* gp;      // P x 3: point gradient
  double* ddiag;   // P x 3: damping diagonal
  PointSummary* summary;  // P
  double* sw;      // optional N: sqrt weight per observation (debug linearization only)
};

// The pose columns of an observation's camera Jacobian (schur/point.rs:286-313), J times the motion
// of the camera point: pose_motion (point.rs:730-762) [-[q]x | s I] at q = RX, or at the camera point
// q = RX + t when the mask holds the translation (the camera turns about its fixed centre);
// translation_motion (point.rs:764-786) alone, s I, when the mask holds the rotation. The FixedBaseline
// camera's translation columns are the baseline times its S^2 tangent basis.
__device__ __forceinline__ void pose_jacobian(const double J[2][3], const double rot[3], const double xc[3],
                                              int mask, int cam, const Gauge& g, double out[2][6]) {
  double m[3][6];
  const double* q = (mask & 2) ? rot : xc;
  const int ts = (mask & 1) ? 3 : 0;  // first translation column
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 6; ++c) m[r][c] = 0.0;
  if (mask & 1) {
    m[0][1] = q[2];
    m[0][2] = -q[1];
    m[1][0] = -q[2];
    m[1][2] = q[0];
    m[2][0] = q[1];
    m[2][1] = -q[0];
  }
  if (mask & 2) {
    if (cam == g.fixed_cam) {
      for (int c = 0; c < 3; ++c) {
        m[c][ts] = g.baseline * g.b0[c];
        m[c][ts + 1] = g.baseline * g.b1[c];
      }
    } else {
      m[0][ts] = g.scene;
      m[1][ts + 1] = g.scene;
      m[2][ts + 2] = g.scene;
    }
  }
  for (int r = 0; r < 2; ++r)
    for (int c = 0; c < 6; ++c) out[r][c] = J[r][0] * m[0][c] + J[r][1] * m[1][c] + J[r][2] * m[2][c];
}

// The point part of the linearization (schur/assembly.rs:893-1040, point_block.rs:78-184): the
// summary, g_p, the scaled gradient norm, the damped factor and its inverse, the damping diagonal,
// the rcond at lambda = 0 and Vhat^-1 g_p.
template <typename T>
__device__ __forceinline__ void point_epilogue(const DevView& v, uint32_t p, const double V[6], const double gp[3],
                                               double cost, double sq, bool ok, double lambda, LinOut<T>& out) {
  PointSummary sm{0, 0, 0, 0, 1.0, 0, 0, 0};
  double* vi = out.vinv + 6 * (size_t)p;
  double* vf = out.vfac + 6 * (size_t)p;
  double* ig = out.ig + 3 * (size_t)p;
  for (int k = 0; k < 6; ++k) vi[k] = vf[k] = 0.0;
  ig[0] = ig[1] = ig[2] = 0.0;
  out.gp[3 * (size_t)p] = gp[0];
  out.gp[3 * (size_t)p + 1] = gp[1];
  out.gp[3 * (size_t)p + 2] = gp[2];
  if (!ok) {
    sm.invalid = 1;
    out.summary[p] = sm;
    return;
  }
  sm.cost = cost;
  sm.sq = sq;
  if (v.fixed_points[p]) {
    out.summary[p] = sm;
    return;
  }
  // scaled_gradient_inf_norm (schur/assembly.rs:1071-1090)
  {
    double scale = fmax(fmax(fmax(0.0, V[0]), V[2]), V[5]);
    double gn;
    if (!(isfinite(scale) && scale > 0.0)) {
      gn = (gp[0] == 0.0 && gp[1] == 0.0 && gp[2] == 0.0) ? 0.0 : INFINITY;
    } else {
      double fl = 64.0 * kEps * scale;
      gn = fmax(fmax(fabs(gp[0]) / sqrt(fmax(V[0], fl)), fabs(gp[1]) / sqrt(fmax(V[2], fl))),
                fabs(gp[2]) / sqrt(fmax(V[5], fl)));
    }
    sm.grad_norm = gn;
  }
  double damped[6], inv[6], fac[6];
  if (!point_factor(V, lambda, damped, inv, fac)) {
    sm.invalid = 1;
    if (lambda == 0.0) {
      sm.weak = 1;
      sm.min_rcond = 0.0;
    }
    out.summary[p] = sm;
    return;
  }
  double dd[3];
  point_damping_diagonal(V, dd);
  out.ddiag[3 * (size_t)p] = dd[0];
  out.ddiag[3 * (size_t)p + 1] = dd[1];
  out.ddiag[3 * (size_t)p + 2] = dd[2];
  if (lambda == 0.0) {
    double rc = point_rcond(V, inv);
    sm.min_rcond = rc;
    if (rc <= 64.0 * kEps * 3.0) sm.weak = 1;
  }
  double igv[3];
  sym3_apply(inv, gp, igv);
  sm.point_red = 0.5 * (gp[0] * igv[0] + gp[1] * igv[1] + gp[2] * igv[2]);
  for (int k = 0; k < 6; ++k) {
    vi[k] = inv[k];
    vf[k] = fac[k];
  }
  ig[0] = igv[0];
  ig[1] = igv[1];
  ig[2] = igv[2];
  out.summary[p] = sm;
}

// ----------------------------------------------------------------------------------------------
// K2: camera-side block reductions (deterministic chunked segmented sums)
// ----------------------------------------------------------------------------------------------
// An entity is (observation, segment): segment 0 = pose columns, 1 = intrinsic columns.
struct BlockTables {
  int nblocks;
  const int* blk_off;        // parameter offset of each block
  const int* blk_dim;        // dimension of each block
  const int* blk_col;        // column of the block inside an observation's 9-column Jacobian (0 or pose dim)
  const int* blk_edge;       // pose blocks: intrinsic block index of the camera's group with dim > 0, else -1
  const uint32_t* ent;       // entity list, block-major: obs * 2 + seg
  const uint32_t* ent_point; // point of each entity (same order)
  int nchunks;
  const int* chunk_block;    // block of each chunk
  const int* chunk_col;      // Jacobian column of the block's segment for every entity of the chunk
  const uint32_t* chunk_begin;  // into ent
  const uint32_t* chunk_end;
  const int* blk_chunk_begin;   // per block: first chunk
  const int* blk_chunk_end;
};

// Assembly record per block: U lower (21), g (6), reduced g (6), diag (6), edge (18), coupling lower (21)
constexpr int kAsmRec = 21 + 6 + 6 + 6 + 18 + 21;

// Scatter block records into the D-vectors (g, reduced g, diag) — one thread per block.
__global__ void k_block_vectors(BlockTables bt, const double* blk_out, double* gfull, double* gred, double* diag,
                                int* clamp_count, double* diag_minmax) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= bt.nblocks) return;
  const double* rec = blk_out + (size_t)kAsmRec * b;
  int o = bt.blk_off[b], d = bt.blk_dim[b];
  double s = 0.0;
  for (int k = 0; k < d; ++k) {
    gfull[o + k] = rec[21 + k];
    gred[o + k] = rec[27 + k];
    s = fmax(s, rec[33 + k]);
  }
  // raw diagonal extrema before clamping (finalize_assembly, schur/assembly.rs:701-712)
  double mn = INFINITY, mx = 0.0;
  for (int k = 0; k < d; ++k) {
    mn = fmin(mn, rec[33 + k]);
    mx = fmax(mx, rec[33 + k]);
  }
  diag_minmax[2 * b] = mn;
  diag_minmax[2 * b + 1] = mx;
  // clamp_damping_block (schur/assembly.rs:744-766)
  double fl = s > 0.0 ? 64.0 * kEps * s : 1.0;
  int cl = 0;
  for (int k = 0; k < d; ++k) {
    double v = rec[33 + k];
    if (v < fl) {
      v = fl;
      ++cl;
    }
    diag[o + k] = v;
  }
  clamp_count[b] = cl;
}

// ----------------------------------------------------------------------------------------------
// Explicit Schur blocks via pair lists (Direct / dense S and cross-pair preconditioner terms)
// ----------------------------------------------------------------------------------------------
struct PairTables {
  int ngroups;
  const int* grp_row;        // row block
  const int* grp_col;        // column block
  const uint32_t* grp_begin; // into pairs
  const uint32_t* grp_end;
  const uint32_t* pair_a;    // entity (obs*2+seg) on the row side
  const uint32_t* pair_b;    // entity on the column side
  const uint32_t* pair_p;    // point
};

// out[g] (36 values, row-major d_row x d_col) = sum over pairs of Jc_a^T (Jp_a Vhat^-1 Jp_b^T) Jc_b
template <typename T>
__global__ void __launch_bounds__(32) k_pairs(PairTables pt, BlockTables bt, LinOut<T> lin, const int* seg_col,
                                              double* out) {
  int gidx = blockIdx.x;
  if (gidx >= pt.ngroups) return;
  int lane = threadIdx.x;
  int rb = pt.grp_row[gidx], cb = pt.grp_col[gidx];
  int dr = bt.blk_dim[rb], dc = bt.blk_dim[cb];
  double acc[36];
#pragma unroll
  for (int k = 0; k < 36; ++k) acc[k] = 0.0;
  for (uint32_t i = pt.grp_begin[gidx] + lane; i < pt.grp_end[gidx]; i += 32) {
    uint32_t ea = pt.pair_a[i], eb = pt.pair_b[i], p = pt.pair_p[i];
    uint32_t oa = ea >> 1, ob = eb >> 1;
    int ca = seg_col[ea], cbcol = seg_col[eb];
    const int rs = lin.rs;
    const T* jpa = lin.rec + lin.obs_rec[oa] + kJp * rs;
    const T* jpb = lin.rec + lin.obs_rec[ob] + kJp * rs;
    const double* vi = lin.vinv + 6 * (size_t)p;
    double pa0[3] = {(double)jpa[0], (double)jpa[rs], (double)jpa[2 * rs]};
    double pa1[3] = {(double)jpa[3 * rs], (double)jpa[4 * rs], (double)jpa[5 * rs]};
    double pb0[3] = {(double)jpb[0], (double)jpb[rs], (double)jpb[2 * rs]};
    double pb1[3] = {(double)jpb[3 * rs], (double)jpb[4 * rs], (double)jpb[5 * rs]};
    double t0[3], t1[3];
    sym3_apply(vi, pb0, t0);
    sym3_apply(vi, pb1, t1);
    double A00 = pa0[0] * t0[0] + pa0[1] * t0[1] + pa0[2] * t0[2];
    double A01 = pa0[0] * t1[0] + pa0[1] * t1[1] + pa0[2] * t1[2];
    double A10 = pa1[0] * t0[0] + pa1[1] * t0[1] + pa1[2] * t0[2];
    double A11 = pa1[0] * t1[0] + pa1[1] * t1[1] + pa1[2] * t1[2];
    const T* ja = lin.rec + lin.obs_rec[oa];
    const T* jb = lin.rec + lin.obs_rec[ob];
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      if (r >= dr) break;
      double a0 = (double)ja[(ca + r) * rs], a1 = (double)ja[(9 + ca + r) * rs];
      double c0 = a0 * A00 + a1 * A10, c1 = a0 * A01 + a1 * A11;
#pragma unroll
      for (int s2 = 0; s2 < 6; ++s2) {
        if (s2 >= dc) break;
        acc[6 * r + s2] += c0 * (double)jb[(cbcol + s2) * rs] + c1 * (double)jb[(9 + cbcol + s2) * rs];
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 36; ++k) {
    double s = warp_sum(acc[k]);
    if (lane == 0) out[(size_t)36 * gidx + k] = s;
  }
}

// ----------------------------------------------------------------------------------------------
// Device-side PCG control (sparse/pcg.rs:23-119). One CTA computes each scalar reduction and, in
// its epilogue, the recurrence coefficient and the loop status, so the PCG iterations run as a
// CUDA graph without host round trips. Every kernel of an iteration returns immediately once the
// status leaves kRunning, so iterations launched past termination cost only their launch.
// ----------------------------------------------------------------------------------------------
enum PcgStatus : int { kRunning = 0, kCheckResidual = 1, kRejected = 2, kExhausted = 3 };
struct PcgCtl {
  // rho_slot: r.z of the current residual, in one of two slots: an iteration reads slot p and its
  // direction kernel writes slot p ^ 1, so no CTA reads a value another CTA of the same kernel writes.
  double n0, rho_slot[2], alpha, beta, curv, rr, rz, ratio, tol;
  int status, terms, max_it, pad;
};

__device__ __forceinline__ bool pcg_stopped(const PcgCtl* ctl) { return ctl && ctl->status != kRunning; }

// Programmatic dependent launch. A kernel launched with programmatic stream serialization may start
// while the kernel before it on the stream is still running: it first issues the loads of data that
// stays constant during the PCG loop, then lets its own successor launch (pdl_trigger) and waits for
// its predecessor to complete with its writes visible (pdl_wait) before it reads anything that
// kernel, or any earlier one, writes. A successor launches only after every CTA of this kernel has
// triggered or exited, so the waits always end. Launched without the attribute, both are no-ops.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Sum of v[0..n) by one warp in a fixed order (lane-strided partial sums, then a shuffle tree); the
// result is valid in lane 0 and identical in every CTA that evaluates it.
__device__ __forceinline__ double warp_fixed_sum(const double* __restrict__ v, int n, int lane) {
  double acc = 0.0;
  for (int i = lane; i < n; i += 32) acc += v[i];
  return warp_sum(acc);
}

// PCG iteration, part 1, after the product q = S d (sparse/pcg.rs:23-119). Every CTA sums the
// finalize's per-CTA curvature terms in the same order, so all agree on alpha; a curvature <= 0
// or a non-finite alpha rejects. Thread per block: x += alpha d, r -= alpha q, z = M^-1 r with the
// Jacobi-scaled Cholesky factor, and the block's |r|^2 and r.z, reduced per CTA in a fixed order.
constexpr int kUpdThreads = 32;  // one warp per CTA: many CTAs, so the blocks' solves spread over the SMs

__global__ void __launch_bounds__(kUpdThreads) k_pcg_update_precond(BlockTables bt, const double* __restrict__ factor,
                                                            const double* __restrict__ dq_part, int ndq,
                                                            const double* __restrict__ d, const double* __restrict__ q,
                                                            double* x, double* r, double* z, double* rr_part,
                                                            double* rz_part, int slot, PcgCtl* ctl) {
  __shared__ double s_alpha;
  __shared__ int s_go;
  const int tid = threadIdx.x, lane = tid & 31;
  // the block's factor (lower 6x6 row-major, then the 6 Jacobi scales; constant during PCG), 16 B
  // loads, before the wait
  const int b = blockIdx.x * blockDim.x + tid;
  const bool have = b < bt.nblocks;
  const int dim = have ? bt.blk_dim[b] : 0, o = have ? bt.blk_off[b] : 0;
  double F[42];
  if (have) {
    const double2* f2 = reinterpret_cast<const double2*>(factor + 42 * (size_t)b);
#pragma unroll
    for (int q = 0; q < 21; ++q) {
      const double2 v = __ldg(f2 + q);
      F[2 * q] = v.x;
      F[2 * q + 1] = v.y;
    }
  }
  pdl_trigger();
  pdl_wait();
  if (ctl->status != kRunning) return;
  // this block's d, q, r and x, requested together with the curvature terms
  double dv[6], qv[6], rv[6], xv[6];
#pragma unroll
  for (int i = 0; i < 6; ++i)
    if (i < dim) {
      dv[i] = d[o + i];
      qv[i] = q[o + i];
      rv[i] = r[o + i];
      xv[i] = x[o + i];
    }
  {
    const double curv = warp_fixed_sum(dq_part, ndq, lane);
    if (lane == 0) {
      s_go = 0;
      double alpha = 0.0;
      if (isfinite(curv) && curv > 0.0) {
        alpha = ctl->rho_slot[slot] / curv;
        if (isfinite(alpha)) s_go = 1;
      }
      s_alpha = alpha;
      if (blockIdx.x == 0) {
        ctl->curv = curv;
        if (s_go)
          ctl->alpha = alpha;
        else
          ctl->status = kRejected;
      }
    }
  }
  __syncthreads();
  if (!s_go) return;
  const double alpha = s_alpha;
  double rr = 0.0, rz = 0.0;
  if (have) {
    double sv[6];
#pragma unroll
    for (int i = 0; i < 6; ++i)
      if (i < dim) {
        x[o + i] = xv[i] + alpha * dv[i];
        rv[i] = rv[i] - alpha * qv[i];
        r[o + i] = rv[i];
      }
    // forward and back substitution, unrolled over the maximum block size (6) so F stays in registers
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      if (i < dim) {
        double v = rv[i] / F[36 + i];
#pragma unroll
        for (int k = 0; k < i; ++k) v -= F[6 * i + k] * sv[k];
        sv[i] = v / F[6 * i + i];
      }
    }
#pragma unroll
    for (int i = 5; i >= 0; --i) {
      if (i < dim) {
        double v = sv[i];
#pragma unroll
        for (int k = i + 1; k < 6; ++k)
          if (k < dim) v -= F[6 * k + i] * sv[k];
        sv[i] = v / F[6 * i + i];
      }
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      if (i < dim) {
        const double zi = sv[i] / F[36 + i];
        z[o + i] = zi;
        rr += rv[i] * rv[i];
        rz += rv[i] * zi;
      }
    }
  }
  rr = warp_sum(rr);
  rz = warp_sum(rz);
  if (tid == 0) {
    rr_part[blockIdx.x] = rr;
    rz_part[blockIdx.x] = rz;
  }
}

// PCG iteration, part 2: every CTA sums the per-CTA |r|^2 and r.z in the same order and takes the
// same decision: the recursive residual ratio at or below the tolerance hands over to the host's
// true-residual check; r.z <= 0 or a non-finite value rejects; otherwise beta = r.z / rho and
// d = z + beta d (also at the iteration limit, which ends the loop after this direction).
__global__ void k_pcg_direction(int n, const double* __restrict__ rr_part, const double* __restrict__ rz_part,
                                int nparts, const double* __restrict__ z, double* d, int slot, PcgCtl* ctl) {
  pdl_trigger();
  pdl_wait();
  if (ctl->status != kRunning && ctl->status != kExhausted) return;
  __shared__ double s_beta;
  __shared__ int s_go;
  const int tid = threadIdx.x, lane = tid & 31;
  const int i = blockIdx.x * blockDim.x + tid;
  double zi = 0.0, di = 0.0;  // requested together with the partial sums
  if (i < n) {
    zi = z[i];
    di = d[i];
  }
  if (tid < 32) {
    const double rr = warp_fixed_sum(rr_part, nparts, lane);
    const double rz = warp_fixed_sum(rz_part, nparts, lane);
    if (lane == 0) {
      const double ratio = sqrt(rr) / ctl->n0;
      int status = kRunning;
      double beta = 0.0;
      if (!isfinite(ratio)) {
        status = kRejected;
      } else if (ratio <= ctl->tol) {
        status = kCheckResidual;
      } else if (!(isfinite(rz) && rz > 0.0)) {
        status = kRejected;
      } else {
        beta = rz / ctl->rho_slot[slot];
        if (!isfinite(beta)) status = kRejected;
      }
      s_go = status == kRunning;
      s_beta = beta;
      if (blockIdx.x == 0) {  // only CTA 0 writes the control block
        const int it = ctl->terms + 1;
        ctl->terms = it;
        ctl->rr = rr;
        ctl->rz = rz;
        ctl->ratio = ratio;
        if (status == kRunning) {
          ctl->beta = beta;
          ctl->rho_slot[slot ^ 1] = rz;
          if (it >= ctl->max_it) status = kExhausted;
        }
        ctl->status = status;
      }
    }
  }
  __syncthreads();
  if (!s_go) return;
  const double beta = s_beta;
  if (i < n) d[i] = zi + beta * di;
}

// ----------------------------------------------------------------------------------------------
// Matrix-free reduced camera system product (implicit Schur)
// ----------------------------------------------------------------------------------------------
}  // namespace omvgba
#include "mv_tiles.cuh"
#include "asm_tiles.cuh"
#include "explicit_s.cuh"
#include "two_view.cuh"
namespace omvgba {

// ----------------------------------------------------------------------------------------------
// K1: the linearization (schur/point.rs:176-448) with one CTA per matvec tile of whole points and
// one thread per observation: project, robust weight, analytic point and camera Jacobians, each
// record component written by a warp as one coalesced line. The per-point sums (V, g_p, cost,
// squared residual) are formed by one thread per point from the observations' row contributions
// staged in shared memory, in track order and row 0 before row 1 (the reference's accumulation
// order, schur/point.rs:388-390), followed by the point epilogue.
// ----------------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(mv_tile_obs<T>(), sizeof(T) == 4 ? 3 : 6) k_linearize_tiles(DevView v, DevState s, Gauge g, LossDev loss,
                                                                      double lambda, LinOut<T> out, MvTiles mt) {
  constexpr int TILE = mv_tile_obs<T>();
  __shared__ double contrib[TILE][2][9];  // per observation and Jacobian row: V (6), g_p (3)
  __shared__ double cs[TILE][2];          // cost, squared residual norm
  __shared__ unsigned char okf[TILE];
  const int t = blockIdx.x, tid = threadIdx.x;
  const uint4 hdr = mt.tile_hdr[t];
  const uint32_t nobs = hdr.x, npt = hdr.y, p0 = hdr.w;
  const unsigned char* slot = mt.slots + (size_t)t * MvSlot::bytes(TILE);
  const uint16_t* poff = reinterpret_cast<const uint16_t*>(slot + MvSlot::poff(TILE));
  const uint16_t* lpt = reinterpret_cast<const uint16_t*>(slot + MvSlot::lpt(TILE));
  const uint32_t o0 = v.pt_off[p0];
  T* rec = out.rec + (size_t)t * TILE * kRec + tid;
  if ((uint32_t)tid < nobs) {
    const uint32_t o = o0 + tid;
    const uint32_t p = p0 + lpt[tid];
    const double X0 = s.points[3 * (size_t)p], X1 = s.points[3 * (size_t)p + 1], X2 = s.points[3 * (size_t)p + 2];
    const int cam = v.obs_cam[o];
    const double* P = s.pose + 12 * cam;
    double rot[3] = {P[0] * X0 + P[1] * X1 + P[2] * X2, P[3] * X0 + P[4] * X1 + P[5] * X2,
                     P[6] * X0 + P[7] * X1 + P[8] * X2};
    double xc[3] = {rot[0] + P[9], rot[1] + P[10], rot[2] + P[11]};
    double r[2], J[2][3], Ji[2][3];
    if (!project_obs(v, s.groups, o, xc, r, J, Ji)) {
      okf[tid] = 0;
#pragma unroll
      for (int k = 0; k < kRec; ++k) rec[k * TILE] = T(0);
      out.rw[2 * (size_t)o] = 0.0;
      out.rw[2 * (size_t)o + 1] = 0.0;
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int k = 0; k < 9; ++k) contrib[tid][a][k] = 0.0;
      cs[tid][0] = cs[tid][1] = 0.0;
    } else {
      okf[tid] = 1;
      const double rn = sqrt(r[0] * r[0] + r[1] * r[1]);
      const double sw = loss.sqrt_weight(rn);
      cs[tid][0] = loss.cost(rn);
      cs[tid][1] = rn * rn;
      double jp[2][3];
      for (int a = 0; a < 2; ++a)
        for (int c = 0; c < 3; ++c) jp[a][c] = (J[a][0] * P[c] + J[a][1] * P[3 + c] + J[a][2] * P[6 + c]) * g.scene;
      for (int a = 0; a < 2; ++a) {
        const double wr = sw * r[a];
        const double w0 = sw * jp[a][0], w1 = sw * jp[a][1], w2 = sw * jp[a][2];
        contrib[tid][a][0] = w0 * w0;
        contrib[tid][a][1] = w1 * w0;
        contrib[tid][a][2] = w1 * w1;
        contrib[tid][a][3] = w2 * w0;
        contrib[tid][a][4] = w2 * w1;
        contrib[tid][a][5] = w2 * w2;
        contrib[tid][a][6] = w0 * wr;
        contrib[tid][a][7] = w1 * wr;
        contrib[tid][a][8] = w2 * wr;
      }
      double jc[2][9];
      for (int a = 0; a < 2; ++a)
        for (int k = 0; k < 9; ++k) jc[a][k] = 0.0;
      const int pd = v.pose_dim[cam];
      if (pd > 0) {
        double pj[2][6];
        pose_jacobian(J, rot, xc, v.pose_mask[cam], cam, g, pj);
        for (int a = 0; a < 2; ++a)
          for (int k = 0; k < pd; ++k) jc[a][k] = pj[a][k];
      }
      if (v.self_cal) {
        const int id = v.intr_dim[v.cam_group[cam]];
        for (int a = 0; a < 2; ++a)
          for (int k = 0; k < id; ++k) jc[a][pd + k] = Ji[a][k];
      }
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int k = 0; k < 9; ++k) rec[(9 * a + k) * TILE] = T(sw * jc[a][k]);
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) rec[(kJp + 3 * a + c) * TILE] = T(sw * jp[a][c]);
      out.rw[2 * (size_t)o] = sw * r[0];
      out.rw[2 * (size_t)o + 1] = sw * r[1];
      if (out.sw) out.sw[o] = sw;
    }
  }
  __syncthreads();
  if ((uint32_t)tid >= npt) return;
  const uint32_t p = p0 + tid;
  double V[6] = {0, 0, 0, 0, 0, 0}, gp[3] = {0, 0, 0};
  double cost = 0.0, sq = 0.0;
  bool ok = true;
  for (uint32_t i = poff[tid]; i < poff[tid + 1]; ++i) {
    if (!okf[i]) {
      ok = false;
      continue;
    }
    cost += cs[i][0];
    sq += cs[i][1];
    for (int a = 0; a < 2; ++a) {
      gp[0] += contrib[i][a][6];
      gp[1] += contrib[i][a][7];
      gp[2] += contrib[i][a][8];
      V[0] += contrib[i][a][0];
      V[1] += contrib[i][a][1];
      V[2] += contrib[i][a][2];
      V[3] += contrib[i][a][3];
      V[4] += contrib[i][a][4];
      V[5] += contrib[i][a][5];
    }
  }
  point_epilogue(v, p, V, gp, cost, sq, ok, lambda, out);
}

// ----------------------------------------------------------------------------------------------
// Block-Jacobi preconditioner (FP64): P_b = U_bb + lambda D_b - C_b - cross pairs
// ----------------------------------------------------------------------------------------------
// PackedCameraBlockFactor::factor (retained/block.rs:171-218): Jacobi-scaled Cholesky of the d x d
// block m into F (36 lower row-major, then the 6 scales); false when it is not positive definite.
__device__ bool camera_block_factor(double m[6][6], int d, double* F) {
  double ds = 0.0;
  for (int i = 0; i < d; ++i) ds = fmax(ds, m[i][i]);
  if (!(isfinite(ds) && ds > 0.0)) return false;
  double fl = 64.0 * kEps * ds;
  double sc[6];
  for (int i = 0; i < d; ++i) sc[i] = sqrt(fmax(m[i][i], fl));
  double L[6][6];
  for (int r = 0; r < d; ++r)
    for (int c = 0; c <= r; ++c) {
      double v = m[r][c] / (sc[r] * sc[c]);
      for (int k = 0; k < c; ++k) v -= L[r][k] * L[c][k];
      if (r == c) {
        if (!(isfinite(v) && v > 64.0 * kEps)) return false;
        L[r][c] = sqrt(v);
      } else {
        L[r][c] = v / L[c][c];
      }
    }
  for (int r = 0; r < 6; ++r)
    for (int c = 0; c < 6; ++c) F[6 * r + c] = (r < d && c <= r) ? L[r][c] : 0.0;
  for (int i = 0; i < 6; ++i) F[36 + i] = i < d ? sc[i] : 1.0;
  return true;
}

__global__ void k_block_factor(BlockTables bt, const double* blk_out, const double* diag, double lambda,
                               const double* cross, const int* blk_cross_begin, const int* blk_cross_end,
                               double* factor, int* fail) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= bt.nblocks) return;
  int d = bt.blk_dim[b], o = bt.blk_off[b];
  const double* rec = blk_out + (size_t)kAsmRec * b;
  double m[6][6];
  int idx = 0;
  for (int r = 0; r < 6; ++r)
    for (int c = 0; c <= r; ++c, ++idx) {
      double v = rec[idx] - rec[57 + idx];
      m[r][c] = v;
      m[c][r] = v;
    }
  for (int g = blk_cross_begin[b]; g < blk_cross_end[b]; ++g) {
    const double* cv = cross + (size_t)36 * g;
    // a diagonal pair group holds each ordered cross pair once: add both orientations
    for (int r = 0; r < d; ++r)
      for (int c = 0; c < d; ++c) m[r][c] -= cv[6 * r + c] + cv[6 * c + r];
  }
  for (int k = 0; k < d; ++k) m[k][k] += lambda * diag[o + k];
  fail[b] = camera_block_factor(m, d, factor + 42 * (size_t)b) ? 0 : 1;
}

// The same block-Jacobi factors from the explicit S: block b's diagonal block of the rows plus
// lambda diag (retained/mod.rs:904-934).
__global__ void k_block_factor_rows(RowTables rt, const double* rows, const double* diag, double lambda,
                                    double* factor, int* fail) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= rt.nblocks) return;
  const int d = rt.blk_dim[b], o = rt.blk_off[b];
  const int s = find_slot(rt.nbr, rt.nbr_begin[b], rt.nbr_begin[b + 1], b);
  double m[6][6];
  for (int r = 0; r < 6; ++r)
    for (int c = 0; c < 6; ++c) m[r][c] = 0.0;
  if (s >= 0) {
    const double* S = rows + rt.slot_off[rt.nbr_begin[b] + s];
    for (int r = 0; r < d; ++r)
      for (int c = 0; c < d; ++c) m[r][c] = S[r * d + c];
  }
  for (int k = 0; k < d; ++k) m[k][k] += lambda * diag[o + k];
  fail[b] = camera_block_factor(m, d, factor + 42 * (size_t)b) ? 0 : 1;
}

__global__ void k_block_precond(BlockTables bt, const double* factor, const double* r, double* z,
                                const PcgCtl* ctl) {
  if (pcg_stopped(ctl)) return;
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= bt.nblocks) return;
  int d = bt.blk_dim[b], o = bt.blk_off[b];
  const double* F = factor + 42 * (size_t)b;
  double s[6];
  for (int i = 0; i < d; ++i) {
    double v = r[o + i] / F[36 + i];
    for (int k = 0; k < i; ++k) v -= F[6 * i + k] * s[k];
    s[i] = v / F[6 * i + i];
  }
  for (int i = d - 1; i >= 0; --i) {
    double v = s[i];
    for (int k = i + 1; k < d; ++k) v -= F[6 * k + i] * s[k];
    s[i] = v / F[6 * i + i];
  }
  for (int i = 0; i < d; ++i) z[o + i] = s[i] / F[36 + i];
}

__global__ void k_axpy2(int n, double alpha, const double* d, const double* q, double* x, double* r) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    x[i] += alpha * d[i];
    r[i] -= alpha * q[i];
  }
}
__global__ void k_xpby(int n, const double* z, double beta, double* d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) d[i] = z[i] + beta * d[i];
}
__global__ void k_neg_copy(int n, const double* a, double* b) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = -a[i];
}
__global__ void k_sub(int n, const double* b, const double* q, double* r) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) r[i] = b[i] - q[i];
}
__global__ void k_axpy(int n, double a, const double* x, double* y) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] += a * x[i];
}
__global__ void k_residual_update(int n, const double* g, const double* q, double* r) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) r[i] = -g[i] - q[i];
}
__global__ void k_scale(int n, double s, double* x) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] *= s;
}

// ----------------------------------------------------------------------------------------------
// K4: step cap, retraction, candidate points
// ----------------------------------------------------------------------------------------------
// Per camera: max of the rotation-part norm and the rest (limit_camera_step, optimizer.rs:677-702)
__global__ void k_step_block_norm(int ncam, const int* pose_off, const int* pose_dim, const double* step,
                                  double* out) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncam) return;
  int d = pose_dim[c], o = pose_off[c];
  if (d == 0) {
    out[c] = 0.0;
    return;
  }
  int fd = d < 3 ? d : 3;
  double s1 = 0.0, s2 = 0.0;
  for (int k = 0; k < fd; ++k) s1 += step[o + k] * step[o + k];
  for (int k = fd; k < d; ++k) s2 += step[o + k] * step[o + k];
  out[c] = fmax(sqrt(s1), sqrt(s2));
}

__host__ __device__ __forceinline__ void exp_so3_dev(const double w[3], double R[9]) {
  // numerics/manifold/so3.rs:254-265 with matrix_polynomial (:420-423)
  double th2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  double th = sqrt(th2);
  double a[3], lin, quad;
  if (th < 1e-10) {
    a[0] = w[0];
    a[1] = w[1];
    a[2] = w[2];
    lin = 1.0;
    quad = 0.5;
  } else {
    a[0] = w[0] / th;
    a[1] = w[1] / th;
    a[2] = w[2] / th;
    lin = sin(th);
    quad = 1.0 - cos(th);
  }
  double K[3][3] = {{0.0, -a[2], a[1]}, {a[2], 0.0, -a[0]}, {-a[1], a[0], 0.0}};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double k2 = K[i][0] * K[0][j] + K[i][1] * K[1][j] + K[i][2] * K[2][j];
      R[3 * i + j] = (i == j ? 1.0 : 0.0) + K[i][j] * lin + k2 * quad;
    }
}

// retract_poses (optimizer.rs:376-424) and retract_cameras (self_calibration/optimizer.rs:565-587)
__global__ void k_retract(DevView v, int ng, const double* step, Gauge g, const double* cur_pose,
                          const double* cur_groups, double* cand_pose, double* cand_groups) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < v.ncam) {
    const double* P = cur_pose + 12 * c;
    double* Q = cand_pose + 12 * c;
    int d = v.pose_dim[c], o = v.pose_off[c];
    const int mask = v.pose_mask[c];
    if (d == 0) {
      for (int k = 0; k < 12; ++k) Q[k] = P[k];
    } else {
      // retract_poses_with_masks (optimizer.rs:442-510); a full mask is retract_poses (:376-424)
      double U[9];
      int ts = 0;
      if (mask & 1) {
        double w[3] = {step[o], step[o + 1], step[o + 2]};
        exp_so3_dev(w, U);
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += U[3 * i + k] * P[3 * k + j];
            Q[3 * i + j] = s;
          }
        ts = 3;
      } else {
        for (int k = 0; k < 9; ++k) Q[k] = P[k];
      }
      if (!(mask & 2)) {  // t' = Exp(w) t keeps the centre -R^T t
        for (int i = 0; i < 3; ++i)
          Q[9 + i] = (mask & 1) ? U[3 * i] * P[9] + U[3 * i + 1] * P[10] + U[3 * i + 2] * P[11] : P[9 + i];
      } else if (c == g.fixed_cam) {
        // retract_s2 (numerics/manifold.rs:133-147)
        double d0 = step[o + ts], d1 = step[o + ts + 1];
        double vv[3] = {g.b0[0] * d0 + g.b1[0] * d1, g.b0[1] * d0 + g.b1[1] * d1, g.b0[2] * d0 + g.b1[2] * d1};
        double th = sqrt(vv[0] * vv[0] + vv[1] * vv[1] + vv[2] * vv[2]);
        double tn = sqrt(g.dir[0] * g.dir[0] + g.dir[1] * g.dir[1] + g.dir[2] * g.dir[2]);
        double tv[3] = {g.dir[0] / tn, g.dir[1] / tn, g.dir[2] / tn};
        double out[3];
        if (th < 1e-10) {
          double s[3] = {tv[0] + vv[0], tv[1] + vv[1], tv[2] + vv[2]};
          double n = sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
          out[0] = s[0] / n;
          out[1] = s[1] / n;
          out[2] = s[2] / n;
        } else {
          double cs = cos(th), sn = sin(th) / th;
          for (int k = 0; k < 3; ++k) out[k] = tv[k] * cs + vv[k] * sn;
        }
        for (int k = 0; k < 3; ++k) Q[9 + k] = g.baseline * out[k];
      } else {
        for (int k = 0; k < 3; ++k) Q[9 + k] = P[9 + k] + g.scene * step[o + ts + k];
      }
    }
  }
  if (v.self_cal && c < ng) {
    const double* G = cur_groups + 3 * c;
    double* H = cand_groups + 3 * c;
    int d = v.intr_dim[c], o = v.intr_off[c];
    double dl[3] = {0, 0, 0};
    for (int k = 0; k < d; ++k) dl[k] = step[o + k];
    if (d == 0) {
      H[0] = G[0];
      H[1] = G[1];
      H[2] = G[2];
    } else {
      H[0] = G[0] * exp(dl[0]);
      H[1] = G[1] + dl[1];
      H[2] = G[2] + dl[2];
    }
  }
}

// Admitted track cost (schur/point.rs:705-728): returns false when a projection fails or the
// geometry is not admitted.
__device__ bool admitted_cost(const DevView& v, const double* pose, const double* groups, const double X[3], int p,
                              const LossDev& loss, double scene, int admission, double* cost) {
  TrackGeometryDev geo;
  geo.init(scene);
  double total = 0.0;
  for (uint32_t o = v.pt_off[p]; o < v.pt_off[p + 1]; ++o) {
    int cam = v.obs_cam[o];
    const double* P = pose + 12 * cam;
    double xc[3];
    for (int i = 0; i < 3; ++i) xc[i] = P[3 * i] * X[0] + P[3 * i + 1] * X[1] + P[3 * i + 2] * X[2] + P[9 + i];
    double r[2], J[2][3], Ji[2][3];
    if (!project_obs(v, groups, o, xc, r, J, Ji)) return false;
    // rotate_transposed(R, camera point)
    double off[3];
    for (int j = 0; j < 3; ++j) off[j] = P[j] * xc[0] + P[3 + j] * xc[1] + P[6 + j] * xc[2];
    geo.push(off[0], off[1], off[2]);
    total += loss.cost(sqrt(r[0] * r[0] + r[1] * r[1]));
  }
  bool ok = admission == 0 ? true : (admission == 1 ? !geo.collapsed() : !geo.degenerate());
  if (!ok) return false;
  *cost = total;
  return true;
}

struct CandidateOut {
  double cost, step_sq, damping, failed;
};

template <typename T>
__global__ void __launch_bounds__(128) k_candidate_points(DevView v, LinOut<T> lin, const double* step,
                                                          DevState cur, DevState cand, Gauge g, LossDev loss,
                                                          RedVec<4>* out) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= v.P) return;
  double X[3] = {cur.points[3 * p], cur.points[3 * p + 1], cur.points[3 * p + 2]};
  RedVec<4> res;
  res.v[0] = res.v[1] = res.v[2] = res.v[3] = 0.0;
  if (v.fixed_points[p]) {
    double c;
    cand.points[3 * p] = X[0];
    cand.points[3 * p + 1] = X[1];
    cand.points[3 * p + 2] = X[2];
    if (!admitted_cost(v, cand.pose, cand.groups, X, p, loss, 0.0, 0, &c))
      res.v[3] = 1.0;
    else
      res.v[0] = c;
    out[p] = res;
    return;
  }
  // back-substitution: dp = -(Vhat^-1 g_p + Vhat^-1 sum_o Jp_o^T Jc_o dc_o)  (schur/point.rs:537-596)
  double b0 = 0, b1 = 0, b2 = 0;
  for (uint32_t o = v.pt_off[p]; o < v.pt_off[p + 1]; ++o) {
    int cam = v.obs_cam[o];
    int pd = v.pose_dim[cam], po = v.pose_off[cam];
    const T* jc = lin.rec + lin.obs_rec[o];
    const int rs = lin.rs;
    double e0 = 0, e1 = 0;
    for (int k = 0; k < pd; ++k) {
      e0 += (double)jc[k * rs] * step[po + k];
      e1 += (double)jc[(9 + k) * rs] * step[po + k];
    }
    if (v.self_cal) {
      int gi = v.cam_group[cam];
      int id = v.intr_dim[gi], io = v.intr_off[gi];
      for (int k = 0; k < id; ++k) {
        e0 += (double)jc[(pd + k) * rs] * step[io + k];
        e1 += (double)jc[(9 + pd + k) * rs] * step[io + k];
      }
    }
    const T* jp = jc + kJp * rs;
    b0 += (double)jp[0] * e0 + (double)jp[3 * rs] * e1;
    b1 += (double)jp[rs] * e0 + (double)jp[4 * rs] * e1;
    b2 += (double)jp[2 * rs] * e0 + (double)jp[5 * rs] * e1;
  }
  const double* vi = lin.vinv + 6 * (size_t)p;
  const double* ig = lin.ig + 3 * (size_t)p;
  double bb[3] = {b0, b1, b2}, z[3];
  sym3_apply(vi, bb, z);
  double sp[3] = {-(ig[0] + z[0]), -(ig[1] + z[1]), -(ig[2] + z[2])};
  double st[3] = {X[0] + g.scene * sp[0], X[1] + g.scene * sp[1], X[2] + g.scene * sp[2]};
  // candidate_rule (point_geometry.rs:110-130)
  double c;
  bool moved = false, have = false;
  if (admitted_cost(v, cand.pose, cand.groups, st, p, loss, g.scene, 2, &c)) {
    moved = true;
    have = true;
  } else if (admitted_cost(v, cand.pose, cand.groups, X, p, loss, g.scene, 1, &c)) {
    have = true;
  } else {
    double c2;
    if (!admitted_cost(v, cur.pose, cur.groups, X, p, loss, g.scene, 1, &c2)) {
      if (admitted_cost(v, cand.pose, cand.groups, X, p, loss, g.scene, 0, &c)) have = true;
    }
  }
  if (!have) {
    res.v[3] = 1.0;
    out[p] = res;
    return;
  }
  const double* P = moved ? st : X;
  cand.points[3 * p] = P[0];
  cand.points[3 * p + 1] = P[1];
  cand.points[3 * p + 2] = P[2];
  res.v[0] = c;
  if (moved) {
    res.v[1] = sp[0] * sp[0] + sp[1] * sp[1] + sp[2] * sp[2];
    const double* dd = lin.ddiag + 3 * (size_t)p;
    res.v[2] = dd[0] * sp[0] * sp[0] + dd[1] * sp[1] * sp[1] + dd[2] * sp[2] * sp[2];
  }
  out[p] = res;
}

// Track-cost metrics at the current state (schur/diagnostics.rs:18-44), per point: cost, squared residual.
__global__ void k_metrics(DevView v, DevState s, LossDev loss, RedVec<3>* out) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= v.P) return;
  RedVec<3> r;
  r.v[0] = r.v[1] = r.v[2] = 0.0;
  double X[3] = {s.points[3 * p], s.points[3 * p + 1], s.points[3 * p + 2]};
  for (uint32_t o = v.pt_off[p]; o < v.pt_off[p + 1]; ++o) {
    const double* P = s.pose + 12 * v.obs_cam[o];
    double xc[3];
    for (int i = 0; i < 3; ++i) xc[i] = P[3 * i] * X[0] + P[3 * i + 1] * X[1] + P[3 * i + 2] * X[2] + P[9 + i];
    double rr[2], J[2][3], Ji[2][3];
    if (!project_obs(v, s.groups, o, xc, rr, J, Ji)) {
      r.v[2] = 1.0;
      continue;
    }
    double rn = sqrt(rr[0] * rr[0] + rr[1] * rr[1]);
    r.v[0] += loss.cost(rn);
    r.v[1] += rn * rn;
  }
  out[p] = r;
}

// Observations whose measurement cannot be inverted (kernel/multi_view/model.rs:350-364).
__global__ void k_noninvertible(DevView v, int N, const double* groups, RedVec<1>* out) {
  int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= N) return;
  double bad = 0.0;
  double mx = v.obs_px[2 * o], my = v.obs_px[2 * o + 1];
  if (v.self_cal) {
    RadialDev c = make_radial(groups + 3 * v.cam_group[v.obs_cam[o]]);
    bad = radial_bearing_ok(c, mx, my) ? 0.0 : 1.0;
  } else if (!v.pixel_model) {
    const FixedCameraDev& m = v.models[v.obs_model[o]];
    bad = m.remove_distortion((mx - m.cx) / m.fx, (my - m.cy) / m.fy) ? 0.0 : 1.0;
  }
  out[o].v[0] = bad;
}

// ----------------------------------------------------------------------------------------------
// Host driver
// ----------------------------------------------------------------------------------------------
static inline int grid_for(size_t n, int threads) { return (int)std::max<size_t>(1, (n + threads - 1) / threads); }

struct Layout {
  int D = 0;
  std::vector<int> pose_off, pose_dim, intr_off, intr_dim;
  std::vector<int> cam_pose_block, group_block;  // block index or -1
};

static Layout make_layout(const NativeProblem& n) {
  Layout L;
  L.pose_off.resize(n.ncam);
  L.pose_dim.resize(n.ncam);
  int off = 0;
  for (int c = 0; c < n.ncam; ++c) {
    int d = pose_block_dim(n, c);
    L.pose_off[c] = off;
    L.pose_dim[c] = d;
    off += d;
  }
  size_t ng = n.self_cal ? n.group_dim.size() : 0;
  L.intr_off.assign(std::max<size_t>(ng, 1), 0);
  L.intr_dim.assign(std::max<size_t>(ng, 1), 0);
  for (size_t g = 0; g < ng; ++g) {
    L.intr_off[g] = off;
    L.intr_dim[g] = n.group_dim[g];
    off += n.group_dim[g];
  }
  L.D = off;
  return L;
}

struct Setup {
  // block tables (host copies)
  std::vector<int> blk_off, blk_dim, blk_col, blk_edge;
  std::vector<uint32_t> blk_ent;          // nb + 1: each block's range in ent
  std::vector<int> cam_block, grp_block;  // parameter block of each camera's pose / each group, or -1
  FillVector<uint32_t> ent, ent_point;  // written completely by the construction
  std::vector<int> chunk_block, chunk_col, blk_chunk_begin, blk_chunk_end;
  std::vector<uint32_t> chunk_begin, chunk_end;
  FillVector<int> seg_col;       // per entity id (obs*2+seg): column (all written)
  // cross same-block pairs (preconditioner)
  std::vector<int> xgrp_row, xgrp_col;
  std::vector<uint32_t> xgrp_begin, xgrp_end, xpair_a, xpair_b, xpair_p;
  std::vector<int> blk_cross_begin, blk_cross_end;
  FillVector<int> ent_block;  // entity (observation * 2 + segment) -> parameter block, -1 when absent
  // explicit S (block rows) and its banded factorization
  std::vector<uint32_t> nbr_begin;  // nb + 1
  std::vector<int> nbr, nbr_row;    // neighbour blocks of each block, ascending, and their row block
  std::vector<uint64_t> slot_off;   // entries + 1
  std::vector<int> perm_off;        // per block: first position in the factorization order
  std::vector<int> perm_to_orig;    // D: parameter at each position of the factorization order
  int bwt = 0, nt = 0;              // band width and side of the factor, in 64 x 64 tiles
  int max_track = 0;                // longest track
  uint64_t max_row = 0;             // longest block row of S (doubles)
};

// Tiles of the fused matvec for one record precision (host tables).
struct TileSet {
  int tile = 0;
  std::vector<uint32_t> tile_hdr;  // 4 per tile: observations, points, segments, first point
  FillVector<unsigned char> slots;  // each tile's body zeroes its own slot first
  std::vector<uint32_t> blk_part;  // nblocks + 1
  FillVector<uint32_t> obs_rec;    // element index of each observation's record component 0 (all written)
};

// Tiles of whole points with at most `tile` observations. A tile's observations are grouped by
// camera into segments (ascending camera, observation order inside); each segment feeds the
// camera's pose block and its intrinsic block. Each block owns a contiguous partial region with one
// dim-wide row per segment that feeds it, in tile order: the fixed order in which the product sums
// a block's partials. The tile's metadata slot (layout in mv_tiles.cuh) holds the per-observation
// segment, local point and segment-order position, the point ranges, and per segment its parameter
// offsets and the rows of its partials.
thread_local unsigned tl_host_threads = 0;  // 0: hardware_concurrency
void set_host_thread_limit(unsigned threads) { tl_host_threads = threads; }
unsigned host_thread_limit() {
  return tl_host_threads ? tl_host_threads : std::max(1u, std::thread::hardware_concurrency());
}

// Runs body(i) for i in [0, count) on up to host_thread_limit() threads, in contiguous ranges. The
// bodies write disjoint outputs, so the result does not depend on the thread count.
template <typename Body>
static void host_parallel_for(size_t count, Body body) {
  const unsigned hw = host_thread_limit();
  const size_t nthreads = std::min<size_t>(hw, count / 64 + 1);
  const size_t per = (count + nthreads - 1) / std::max<size_t>(nthreads, 1);
  auto run = [&](size_t k) {
    const size_t b = std::min(count, k * per), e = std::min(count, b + per);
    for (size_t i = b; i < e; ++i) body(i);
  };
  std::vector<std::thread> pool;
  for (size_t k = 1; k < nthreads; ++k) pool.emplace_back(run, k);
  run(0);
  for (auto& t : pool) t.join();
}

// Runs body(chunk, begin, end) over [0, count) cut into `chunks` contiguous ranges of equal size (the
// last shorter), on up to host_thread_limit() threads. Callers that combine per-chunk results do so
// in chunk order, so the result does not depend on the thread count.
template <typename Body>
static void host_parallel_chunks(size_t count, size_t chunks, Body body) {
  const size_t per = (count + chunks - 1) / std::max<size_t>(chunks, 1);
  const unsigned hw = host_thread_limit();
  const size_t nthreads = std::min<size_t>(std::min<size_t>(hw, chunks), count / 65536 + 1);
  std::atomic<size_t> next{0};
  auto worker = [&]() {
    for (size_t c; (c = next.fetch_add(1)) < chunks;) {
      const size_t b = std::min(count, c * per), e = std::min(count, b + per);
      body(c, b, e);
    }
  };
  std::vector<std::thread> pool;
  for (size_t i = 1; i < nthreads; ++i) pool.emplace_back(worker);
  worker();
  for (auto& t : pool) t.join();
}

static void build_tiles(const NativeProblem& n, const Layout& L, const Setup& setup, int tile, TileSet& S) {
  const auto& ent_block = setup.ent_block;
  const int nblocks = (int)setup.blk_off.size();
  const size_t slot_bytes = MvSlot::bytes(tile);
  S.tile = tile;
  size_t P = n.points.size() / 3;
  S.obs_rec.resize(n.obs_cam.size());  // every observation lies in exactly one tile
  struct SegRef {
    uint32_t tile, s;
    int bp, bi;
  };
  // whole points, in order, packed greedily into tiles of at most `tile` observations
  std::vector<std::pair<uint32_t, uint32_t>> range;  // each tile's points [first, end)
  for (size_t p = 0; p < P;) {
    size_t p0 = p;
    uint64_t o0 = n.pt_off[p];
    while (p < P && p - p0 < (size_t)tile && (n.pt_off[p + 1] - o0 <= (uint64_t)tile || p == p0)) ++p;
    if (n.pt_off[p] - o0 > (uint64_t)tile) throw SolveFailure{2, "a point track is longer than the matvec tile"};
    if ((range.size() + 1) * (size_t)tile * kRec >= (1ull << 32))
      throw SolveFailure{3, "record storage exceeds 2^32 elements"};
    range.push_back({(uint32_t)p0, (uint32_t)p});
  }
  const size_t ntiles = range.size();
  S.slots.resize(ntiles * slot_bytes);
  S.tile_hdr.assign(4 * ntiles, 0);
  // each tile's slot, independently; its segments' blocks are kept for the partial regions
  std::vector<std::vector<SegRef>> tile_segs(ntiles);
  host_parallel_for(ntiles, [&](size_t t) {
    std::vector<std::pair<uint32_t, uint16_t>> by_cam;
    std::vector<SegRef>& segs = tile_segs[t];
    const size_t p0 = range[t].first, p = range[t].second;
    const uint64_t o0 = n.pt_off[p0], o1 = n.pt_off[p];
    const uint32_t nobs = (uint32_t)(o1 - o0), npt = (uint32_t)(p - p0);
    unsigned char* B = S.slots.data() + t * slot_bytes;
    std::memset(B, 0, slot_bytes);  // unused rows and padding stay zero
    uint32_t* w0 = reinterpret_cast<uint32_t*>(B + MvSlot::w0(tile));
    uint32_t* w1 = reinterpret_cast<uint32_t*>(B + MvSlot::w1(tile));
    uint16_t* segb = reinterpret_cast<uint16_t*>(B + MvSlot::segb(tile));
    uint16_t* oseg = reinterpret_cast<uint16_t*>(B + MvSlot::oseg(tile));
    uint16_t* lpt = reinterpret_cast<uint16_t*>(B + MvSlot::lpt(tile));
    uint16_t* pos = reinterpret_cast<uint16_t*>(B + MvSlot::pos(tile));
    uint16_t* poff = reinterpret_cast<uint16_t*>(B + MvSlot::poff(tile));
    for (size_t q = p0; q < p; ++q) {
      poff[q - p0] = (uint16_t)(n.pt_off[q] - o0);
      for (uint64_t o = n.pt_off[q]; o < n.pt_off[q + 1]; ++o) lpt[o - o0] = (uint16_t)(q - p0);
    }
    poff[npt] = (uint16_t)nobs;
    by_cam.clear();
    for (uint64_t o = o0; o < o1; ++o) by_cam.push_back({n.obs_cam[o], (uint16_t)(o - o0)});
    std::stable_sort(by_cam.begin(), by_cam.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    uint32_t nseg = 0;
    size_t i = 0;
    while (i < by_cam.size()) {
      size_t j = i;
      while (j < by_cam.size() && by_cam[j].first == by_cam[i].first) ++j;
      const int c = (int)by_cam[i].first;
      const uint64_t o_any = o0 + by_cam[i].second;
      const int pose_b = ent_block[2 * o_any], intr_b = ent_block[2 * o_any + 1];
      uint32_t iw = 0;
      if (n.self_cal) {
        const int g = n.cam_group[c];
        iw = (uint32_t)L.intr_off[g] | ((uint32_t)L.intr_dim[g] << 28);
      }
      w0[nseg] = (uint32_t)L.pose_off[c] | ((uint32_t)L.pose_dim[c] << 28);
      w1[nseg] = iw;
      segb[nseg] = (uint16_t)i;
      for (size_t k = i; k < j; ++k) {
        pos[by_cam[k].second] = (uint16_t)k;
        oseg[by_cam[k].second] = (uint16_t)nseg;
      }
      segs.push_back({(uint32_t)t, nseg, pose_b, intr_b});
      ++nseg;
      i = j;
    }
    segb[nseg] = (uint16_t)nobs;
    for (uint64_t o = o0; o < o1; ++o) S.obs_rec[o] = (uint32_t)(t * (size_t)tile * kRec + (o - o0));
    uint32_t* hdr = &S.tile_hdr[4 * t];
    hdr[0] = nobs;
    hdr[1] = npt;
    hdr[2] = nseg;
    hdr[3] = (uint32_t)p0;
  });
  // partial regions: block b's rows follow the blocks before it; segment rows in tile order
  std::vector<uint32_t> blk_count(nblocks, 0);
  for (const auto& segs : tile_segs)
    for (const SegRef& sr : segs) {
      if (sr.bp >= 0) blk_count[sr.bp]++;
      if (sr.bi >= 0) blk_count[sr.bi]++;
    }
  S.blk_part.assign(nblocks + 1, 0);
  uint64_t total = 0;
  for (int b = 0; b < nblocks; ++b) {
    S.blk_part[b] = (uint32_t)total;
    total += (uint64_t)blk_count[b] * (uint64_t)setup.blk_dim[b];
  }
  if (total >= kNoPartial) throw SolveFailure{3, "matvec partial storage exceeds 2^32 elements"};
  S.blk_part[nblocks] = (uint32_t)total;
  std::vector<uint32_t> next(nblocks, 0);
  for (const auto& segs : tile_segs)
    for (const SegRef& sr : segs) {
      unsigned char* B = S.slots.data() + sr.tile * slot_bytes;
      uint32_t* dpose = reinterpret_cast<uint32_t*>(B + MvSlot::dpose(tile));
      uint32_t* dintr = reinterpret_cast<uint32_t*>(B + MvSlot::dintr(tile));
      dpose[sr.s] = kNoPartial;
      dintr[sr.s] = kNoPartial;
      if (sr.bp >= 0) dpose[sr.s] = S.blk_part[sr.bp] + next[sr.bp]++ * (uint32_t)setup.blk_dim[sr.bp];
      if (sr.bi >= 0) dintr[sr.s] = S.blk_part[sr.bi] + next[sr.bi]++ * (uint32_t)setup.blk_dim[sr.bi];
    }
}

static void build_tables(const NativeProblem& n, const Layout& L, Setup& S) {
  size_t N = n.obs_cam.size(), P = n.points.size() / 3;
  // blocks: pose blocks (camera order) then intrinsic blocks (group order)
  std::vector<int> cam_block(n.ncam, -1), grp_block(L.intr_dim.size(), -1);
  for (int c = 0; c < n.ncam; ++c)
    if (L.pose_dim[c] > 0) {
      cam_block[c] = (int)S.blk_off.size();
      S.blk_off.push_back(L.pose_off[c]);
      S.blk_dim.push_back(L.pose_dim[c]);
      S.blk_col.push_back(0);
      S.blk_edge.push_back(-1);
    }
  if (n.self_cal)
    for (size_t g = 0; g < n.group_dim.size(); ++g)
      if (L.intr_dim[g] > 0) {
        grp_block[g] = (int)S.blk_off.size();
        S.blk_off.push_back(L.intr_off[g]);
        S.blk_dim.push_back(L.intr_dim[g]);
        S.blk_col.push_back(-1);  // column depends on the observation's camera pose dim
        S.blk_edge.push_back(-1);
      }
  if (n.self_cal)
    for (int c = 0; c < n.ncam; ++c)
      if (cam_block[c] >= 0 && grp_block[n.cam_group[c]] >= 0) S.blk_edge[cam_block[c]] = grp_block[n.cam_group[c]];
  int nb = (int)S.blk_off.size();
  S.cam_block = cam_block;
  S.grp_block = grp_block;
  // entity lists per block (stable in observation order)
  // every entry is written below (-1: no block, column 0 and no intrinsic when absent)
  S.seg_col.resize(2 * N);
  FillVector<int> ent_block(2 * N);
  host_parallel_chunks(N, 64, [&](size_t, size_t b, size_t e) {
    for (size_t o = b; o < e; ++o) {
      int c = n.obs_cam[o];
      int pd = L.pose_dim[c];
      ent_block[2 * o] = cam_block[c];  // -1 when the pose has no block
      S.seg_col[2 * o] = 0;
      int intr_b = -1, intr_col = 0;
      if (n.self_cal) {
        int g = n.cam_group[c];
        if (grp_block[g] >= 0) {
          intr_b = grp_block[g];
          intr_col = pd;
        }
      }
      ent_block[2 * o + 1] = intr_b;
      S.seg_col[2 * o + 1] = intr_col;
    }
  });
  // each block's entities in entity order (a stable counting sort): per-chunk counts of every block,
  // ranges laid out block by block and, inside a block, chunk by chunk; then each chunk fills its own
  constexpr size_t kEntChunks = 64;
  const size_t E = 2 * N;
  std::vector<uint32_t> chunk_count(kEntChunks * (size_t)nb, 0);
  host_parallel_chunks(E, kEntChunks, [&](size_t c, size_t b, size_t e) {
    uint32_t* cc = &chunk_count[c * (size_t)nb];
    for (size_t i = b; i < e; ++i)
      if (ent_block[i] >= 0) cc[ent_block[i]]++;
  });
  std::vector<uint32_t> counts(nb + 1, 0);
  std::vector<uint32_t> chunk_at(kEntChunks * (size_t)nb, 0);
  {
    uint32_t at = 0;
    for (int b = 0; b < nb; ++b) {
      counts[b] = at;
      for (size_t c = 0; c < kEntChunks; ++c) {
        chunk_at[c * (size_t)nb + b] = at;
        at += chunk_count[c * (size_t)nb + b];
      }
    }
    counts[nb] = at;
  }
  S.blk_ent = counts;
  S.ent.resize(counts[nb]);  // the fill below writes every position
  S.ent_point.resize(counts[nb]);
  FillVector<uint32_t> obs_point(N);
  host_parallel_chunks(P, 64, [&](size_t, size_t b, size_t e) {
    for (size_t p = b; p < e; ++p)
      for (uint64_t o = n.pt_off[p]; o < n.pt_off[p + 1]; ++o) obs_point[o] = (uint32_t)p;
  });
  host_parallel_chunks(E, kEntChunks, [&](size_t c, size_t b, size_t e) {
    uint32_t* fill = &chunk_at[c * (size_t)nb];
    for (size_t i = b; i < e; ++i) {
      const int blk = ent_block[i];
      if (blk < 0) continue;
      const uint32_t at = fill[blk]++;
      S.ent[at] = (uint32_t)i;
      S.ent_point[at] = obs_point[i >> 1];
    }
  });
  // intrinsic blocks have a per-observation column: stored via seg_col; blk_col = -1 means "use seg".
  // Inside such a block the entities are grouped by column (cameras with pose dims 0, 5, 6), stably,
  // so that every chunk has one column.
  host_parallel_for((size_t)nb, [&](size_t b) {
    if (S.blk_col[b] >= 0) return;
    std::stable_sort(S.ent.begin() + counts[b], S.ent.begin() + counts[b + 1],
                     [&](uint32_t a, uint32_t c) { return S.seg_col[a] < S.seg_col[c]; });
    for (uint32_t i = counts[b]; i < counts[b + 1]; ++i) S.ent_point[i] = obs_point[S.ent[i] >> 1];
  });
  // chunks (never mixing columns)
  S.blk_chunk_begin.assign(nb, 0);
  S.blk_chunk_end.assign(nb, 0);
  for (int b = 0; b < nb; ++b) {
    S.blk_chunk_begin[b] = (int)S.chunk_block.size();
    uint32_t i = counts[b];
    while (i < counts[b + 1]) {
      int col = S.seg_col[S.ent[i]];
      uint32_t j = i;
      while (j < counts[b + 1] && j - i < (uint32_t)kChunk && S.seg_col[S.ent[j]] == col) ++j;
      S.chunk_block.push_back(b);
      S.chunk_col.push_back(col);
      S.chunk_begin.push_back(i);
      S.chunk_end.push_back(j);
      i = j;
    }
    S.blk_chunk_end[b] = (int)S.chunk_block.size();
  }
  // pair lists
  S.blk_cross_begin.assign(nb, 0);
  S.blk_cross_end.assign(nb, 0);
  struct Pair {
    int rb, cb;
    uint32_t p, a, b;
  };
  // per point, in point order; point ranges run in parallel into their own lists, joined in order
  constexpr size_t kPairChunks = 64;
  std::vector<std::vector<Pair>> chunk_xpairs(kPairChunks);
  host_parallel_chunks(P, kPairChunks, [&](size_t c, size_t pb, size_t pe) {
    std::vector<Pair>& xpairs = chunk_xpairs[c];
    std::vector<uint32_t> ents;
    std::vector<int64_t> seen_at(nb, -1);  // point that last used each block (the same-block test)
    for (size_t p = pb; p < pe; ++p) {
      if (n.fixed_points[p]) continue;
      ents.clear();
      bool shared = false;
      for (uint64_t o = n.pt_off[p]; o < n.pt_off[p + 1]; ++o)
        for (int sgm = 0; sgm < 2; ++sgm)
          if (ent_block[2 * o + sgm] >= 0) {
            ents.push_back((uint32_t)(2 * o + sgm));
            int64_t& s = seen_at[ent_block[2 * o + sgm]];
            shared = shared || s == (int64_t)p;
            s = (int64_t)p;
          }
      // only same-block pairs are kept: none when every block of the point is distinct
      if (!shared) continue;
      for (size_t i = 0; i < ents.size(); ++i)
        for (size_t j = 0; j <= i; ++j) {
          uint32_t a = ents[i], b = ents[j];
          int ba = ent_block[a], bb = ent_block[b];
          if (ba < bb) {
            std::swap(a, b);
            std::swap(ba, bb);
          }
          if (ba == bb && a != b) xpairs.push_back({ba, bb, (uint32_t)p, a, b});
        }
    }
  });
  std::vector<Pair> xpairs;
  for (size_t c = 0; c < kPairChunks; ++c) xpairs.insert(xpairs.end(), chunk_xpairs[c].begin(), chunk_xpairs[c].end());
  auto build = [&](std::vector<Pair>& v, std::vector<int>& gr, std::vector<int>& gc, std::vector<uint32_t>& gb,
                   std::vector<uint32_t>& ge, std::vector<uint32_t>& pa, std::vector<uint32_t>& pbv,
                   std::vector<uint32_t>& pp) {
    std::stable_sort(v.begin(), v.end(), [](const Pair& x, const Pair& y) {
      return x.rb != y.rb ? x.rb < y.rb : (x.cb != y.cb ? x.cb < y.cb : false);
    });
    size_t i = 0;
    while (i < v.size()) {
      size_t j = i;
      while (j < v.size() && v[j].rb == v[i].rb && v[j].cb == v[i].cb) ++j;
      gr.push_back(v[i].rb);
      gc.push_back(v[i].cb);
      gb.push_back((uint32_t)i);
      ge.push_back((uint32_t)j);
      i = j;
    }
    pa.resize(v.size());
    pbv.resize(v.size());
    pp.resize(v.size());
    for (size_t k = 0; k < v.size(); ++k) {
      pa[k] = v[k].a;
      pbv[k] = v[k].b;
      pp[k] = v[k].p;
    }
  };
  build(xpairs, S.xgrp_row, S.xgrp_col, S.xgrp_begin, S.xgrp_end, S.xpair_a, S.xpair_b, S.xpair_p);
  for (size_t gidx = 0; gidx < S.xgrp_row.size(); ++gidx) {
    int b = S.xgrp_row[gidx];
    if (S.blk_cross_end[b] == 0 && S.blk_cross_begin[b] == 0) S.blk_cross_begin[b] = (int)gidx;
    S.blk_cross_end[b] = (int)gidx + 1;
  }
  for (int b = 0; b < nb; ++b)
    if (S.blk_cross_end[b] == 0) S.blk_cross_begin[b] = 0;
  S.ent_block = std::move(ent_block);
}

// Neighbour lists of the explicit S (every block Y that shares a point with block X, X included,
// ascending), the offsets of the row blocks, and the factorization order: each camera's pose block,
// then the intrinsic blocks whose first camera it is (cameras in native order), which makes the
// reduced system of a survey banded. bwt is the band of the factor in tiles.
static void build_explicit(const NativeProblem& n, const Layout& L, Setup& S) {
  const int nb = (int)S.blk_off.size();
  const size_t P = n.points.size() / 3;
  S.max_track = 0;
  for (size_t p = 0; p < P; ++p) S.max_track = std::max<int>(S.max_track, (int)(n.pt_off[p + 1] - n.pt_off[p]));
  std::vector<std::vector<int>> nbrs(nb);
  // blocks in contiguous ranges, one per host thread, each with its own marker array; every block's
  // list depends only on the topology
  const size_t nthreads = std::max<size_t>(1, std::min<size_t>(host_thread_limit(), (size_t)nb / 8 + 1));
  const size_t per = ((size_t)nb + nthreads - 1) / nthreads;
  auto run = [&](size_t k) {
    const size_t b0 = std::min((size_t)nb, k * per), b1 = std::min((size_t)nb, b0 + per);
    std::vector<int> stamp(nb, -1);
    for (size_t X = b0; X < b1; ++X) {
      std::vector<int>& out = nbrs[X];
      for (uint32_t i = S.blk_ent[X]; i < S.blk_ent[X + 1]; ++i) {
        const uint32_t p = S.ent_point[i];
        for (uint64_t o = n.pt_off[p]; o < n.pt_off[p + 1]; ++o)
          for (int sg = 0; sg < 2; ++sg) {
            const int Y = S.ent_block[2 * o + sg];
            if (Y >= 0 && stamp[Y] != (int)X) {
              stamp[Y] = (int)X;
              out.push_back(Y);
            }
          }
      }
      std::sort(out.begin(), out.end());
    }
  };
  {
    std::vector<std::thread> pool;
    for (size_t k = 1; k < nthreads; ++k) pool.emplace_back(run, k);
    run(0);
    for (auto& t : pool) t.join();
  }
  S.nbr_begin.assign(nb + 1, 0);
  for (int X = 0; X < nb; ++X) S.nbr_begin[X + 1] = S.nbr_begin[X] + (uint32_t)nbrs[X].size();
  const size_t E = S.nbr_begin[nb];
  S.nbr.resize(E);
  S.nbr_row.resize(E);
  S.slot_off.assign(E + 1, 0);
  uint64_t off = 0;
  for (int X = 0; X < nb; ++X)
    for (size_t k = 0; k < nbrs[X].size(); ++k) {
      const size_t q = S.nbr_begin[X] + k;
      S.nbr[q] = nbrs[X][k];
      S.nbr_row[q] = X;
      S.slot_off[q] = off;
      off += (uint64_t)S.blk_dim[X] * (uint64_t)S.blk_dim[nbrs[X][k]];
    }
  S.slot_off[E] = off;
  S.max_row = 0;
  for (int X = 0; X < nb; ++X)
    S.max_row = std::max<uint64_t>(S.max_row, S.slot_off[S.nbr_begin[X + 1]] - S.slot_off[S.nbr_begin[X]]);
  // factorization order
  std::vector<int> order;
  order.reserve(nb);
  std::vector<int> home(S.grp_block.size(), -1);
  if (n.self_cal)
    for (int c = n.ncam - 1; c >= 0; --c) home[n.cam_group[c]] = c;
  std::vector<std::vector<int>> groups_at(std::max(1, n.ncam));
  std::vector<int> homeless;
  for (size_t g = 0; g < S.grp_block.size(); ++g)
    if (S.grp_block[g] >= 0) {
      if (home[g] >= 0)
        groups_at[home[g]].push_back(S.grp_block[g]);
      else
        homeless.push_back(S.grp_block[g]);
    }
  for (int c = 0; c < n.ncam; ++c) {
    if (S.cam_block[c] >= 0) order.push_back(S.cam_block[c]);
    for (int b : groups_at[c]) order.push_back(b);
  }
  for (int b : homeless) order.push_back(b);
  S.perm_off.assign(nb, 0);
  S.perm_to_orig.assign(L.D, 0);
  int pos = 0;
  for (int b : order) {
    S.perm_off[b] = pos;
    for (int k = 0; k < S.blk_dim[b]; ++k) S.perm_to_orig[pos + k] = S.blk_off[b] + k;
    pos += S.blk_dim[b];
  }
  S.nt = (L.D + kCT - 1) / kCT;
  int bwt = 0;
  for (int X = 0; X < nb; ++X)
    for (uint32_t q = S.nbr_begin[X]; q < S.nbr_begin[X + 1]; ++q) {
      const int Y = S.nbr[q];
      if (S.perm_off[Y] > S.perm_off[X]) continue;
      bwt = std::max(bwt, (S.perm_off[X] + S.blk_dim[X] - 1) / kCT - S.perm_off[Y] / kCT);
    }
  // at least one tile below the diagonal, so a block that straddles a tile boundary stays inside
  S.bwt = std::min(std::max(bwt, 1), std::max(0, S.nt - 1));
}

// Entries of the lower triangle of S (diagonal blocks included) in the block pattern, and the cross
// rows of the point caches: per point, one 3-vector per distinct free camera parameter it touches.
static void pattern_counts(const NativeProblem& n, const Layout& L, const Setup& S, uint64_t* nnz_lower,
                           uint64_t* cross_rows) {
  uint64_t nnz = 0;
  const int nb = (int)S.blk_off.size();
  for (int X = 0; X < nb; ++X) {
    const uint64_t dX = (uint64_t)S.blk_dim[X];
    for (uint32_t q = S.nbr_begin[X]; q < S.nbr_begin[X + 1]; ++q) {
      const int Y = S.nbr[q];
      if (Y < X) nnz += dX * (uint64_t)S.blk_dim[Y];
      if (Y == X) nnz += dX * (dX + 1) / 2;
    }
  }
  uint64_t rows = 0;
  const size_t P = n.points.size() / 3;
  std::vector<uint32_t> groups;
  for (size_t p = 0; p < P; ++p) {
    groups.clear();
    for (uint64_t o = n.pt_off[p]; o < n.pt_off[p + 1]; ++o) {
      const int c = (int)n.obs_cam[o];
      rows += (uint64_t)L.pose_dim[c];
      if (n.self_cal) {
        const uint32_t g = n.cam_group[c];
        if (std::find(groups.begin(), groups.end(), g) == groups.end()) {
          groups.push_back(g);
          rows += (uint64_t)L.intr_dim[g];
        }
      }
    }
  }
  *nnz_lower = nnz;
  *cross_rows = rows;
}

// The budget's automatic choice between the direct and the iterative step (SparseWorkspaceMemoryBudget
// with AUTO_BYTES = 1 GiB unless an explicit budget is given, api.rs:43-52; select_calibrated /
// select_self_calibrating, execution_policy.rs:122-214): the direct estimate is four values per entry
// of the lower reduced pattern plus the point caches (execution_policy.rs:101-120, 66-97), the cached
// retained estimate the point caches plus the camera-space vectors; the direct step must fit 4/5 of
// the budget (execution_policy.rs:279-285). A calibrated problem with at least 250,000 observations
// and D >= 768 prefers the retained PCG when it fits (execution_policy.rs:21-22, 139-148).
static bool auto_prefers_direct(bool self_cal, uint64_t observations, int D, uint64_t points, uint64_t nnz_lower,
                                uint64_t cross_rows, uint64_t budget, uint64_t* direct_out, uint64_t* cached_out) {
  const uint64_t limit = budget ? budget : (uint64_t(1) << 30);
  const uint64_t point_cache = (points + 1) * 8 + points * (1 + 2 * 24) + cross_rows * 24;
  const uint64_t direct = nnz_lower * 8 * 4 + point_cache;
  const uint64_t cached = point_cache + (uint64_t)D * (5 * 8 + 8);
  *direct_out = direct;
  *cached_out = cached;
  const uint64_t guarded = limit / 5 * 4 + limit % 5 * 4 / 5;
  const bool direct_fits = direct <= guarded;
  if (self_cal) return direct_fits;
  if (observations >= 250000 && D >= 768 && cached <= limit) return false;
  return direct_fits;
}

uint64_t fnv1a(const void* data, size_t bytes, uint64_t h) {
  const unsigned char* c = static_cast<const unsigned char*>(data);
  for (size_t i = 0; i < bytes; ++i) h = (h ^ c[i]) * 1099511628211ull;
  return h;
}

uint64_t setup_digest(const NativeProblem& n, const LmOptions& opt) {
  const Layout L = make_layout(n);
  const bool direct = !opt.iterative;
  Setup S;
  build_tables(n, L, S);
  build_explicit(n, L, S);
  TileSet T;
  const bool mixed = opt.precision == 1 && !direct;
  build_tiles(n, L, S, mixed ? mv_tile_obs<float>() : mv_tile_obs<double>(), T);
  uint64_t h = 1469598103934665603ull;
  auto add = [&](const auto& v) { h = fnv1a(v.data(), v.size() * sizeof(v[0]), h); };
  for (const auto* v : {&S.blk_off, &S.blk_dim, &S.blk_col, &S.blk_edge, &S.chunk_block, &S.chunk_col,
                        &S.blk_chunk_begin, &S.blk_chunk_end, &S.xgrp_row, &S.xgrp_col,
                        &S.blk_cross_begin, &S.blk_cross_end})
    add(*v);
  add(S.seg_col);
  add(S.ent_block);
  add(S.blk_ent);
  add(S.nbr_begin);
  add(S.nbr);
  add(S.slot_off);
  add(S.perm_off);
  add(S.perm_to_orig);
  h = fnv1a(&S.bwt, sizeof(S.bwt), h);
  add(S.ent);
  add(S.ent_point);
  add(T.obs_rec);
  for (const auto* v : {&S.chunk_begin, &S.chunk_end, &S.xgrp_begin, &S.xgrp_end, &S.xpair_a, &S.xpair_b, &S.xpair_p,
                        &T.tile_hdr, &T.blk_part})
    add(*v);
  add(T.slots);
  return h;
}

ExecutionPlan execution_plan(const NativeProblem& n, const LmOptions& opt) {
  const Layout L = make_layout(n);
  Setup S;
  build_tables(n, L, S);
  build_explicit(n, L, S);
  ExecutionPlan plan;
  uint64_t nnz = 0, rows = 0;
  pattern_counts(n, L, S, &nnz, &rows);
  const bool direct = auto_prefers_direct(n.self_cal, n.obs_cam.size(), L.D, n.points.size() / 3, nnz, rows,
                                          opt.workspace_budget, &plan.direct_estimate, &plan.cached_estimate);
  // a translation-only solve resolves Auto to the direct solver (native/mod.rs:398-407)
  plan.iterative =
      opt.linear_solver == 0 ? (!direct && !(!n.self_cal && !n.angular && n.translation_only)) : opt.iterative;
  return plan;
}

// Positive-definiteness certificate of a symmetric matrix from its lower-triangle entries: the entries
// are scattered into the banded tile layout of the explicit reduced camera system (bandwidth from the
// entries themselves) and factored by the same tiled Cholesky kernels; the status word says whether
// every pivot was positive.
bool device_certify_positive_definite(Context* ctx, int n, const std::vector<int>& rows, const std::vector<int>& cols,
                                      const std::vector<double>& values) {
  if (n <= 0) return true;
  CUDA_OK(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  int bwt = 0;
  for (size_t q = 0; q < rows.size(); ++q) bwt = std::max(bwt, rows[q] / kCT - cols[q] / kCT);
  const int nt = (n + kCT - 1) / kCT;
  bwt = std::min(std::max(bwt, 1), std::max(nt - 1, 1));
  const size_t count = (size_t)nt * (bwt + 1) * kCTT;
  if (sizeof(double) * count > (size_t(16) << 30))
    throw SolveFailure{3, "the banded factor of the probe's camera system exceeds 16 GiB"};
  DBuf<double> tiles, winv, vals;
  DBuf<int> d_rows, d_cols, status;
  tiles.alloc(count, st);
  winv.alloc((size_t)nt * kCTT, st);
  status.alloc(1, st);
  d_rows.upload(rows.data(), rows.size(), st);
  d_cols.upload(cols.data(), cols.size(), st);
  vals.upload(values.data(), values.size(), st);
  CUDA_OK(cudaFuncSetAttribute(k_tile_trsm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsmSmem));
  CUDA_OK(cudaFuncSetAttribute(k_tile_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUpdateSmem));
  CUDA_OK(cudaMemsetAsync(tiles.p, 0, sizeof(double) * count, st));
  OMVGBA_LAUNCH(k_set_int, 1, 1, 0, st, status.p, 1);
  TileBand tb{n, nt, bwt, tiles.p, winv.p};
  if (!rows.empty())
    OMVGBA_LAUNCH(k_triplets_to_tiles, grid_for(rows.size(), 256), 256, 0, st, (uint32_t)rows.size(), d_rows.p,
                  d_cols.p, vals.p, tb);
  OMVGBA_LAUNCH(k_tiles_pad, 1, kCT, 0, st, tb);
  for (int k = 0; k < nt; ++k) {
    OMVGBA_LAUNCH(k_tile_potrf, 1, 256, 0, st, tb, k, status.p);
    const int m = std::min(bwt, nt - 1 - k);
    if (m > 0) {
      OMVGBA_LAUNCH(k_tile_trsm, m, 256, kTrsmSmem, st, tb, k, status.p);
      OMVGBA_LAUNCH(k_tile_update, m * (m + 1) / 2, 256, kUpdateSmem, st, tb, k, status.p);
    }
  }
  CUDA_OK(cudaGetLastError());
  int ok = 0;
  CUDA_OK(cudaMemcpyAsync(&ok, status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaStreamSynchronize(st));
  return ok != 0;
}

// Device copy of a TileSet plus the fused-matvec launch shape.
struct TileSetDev {
  DBuf<uint32_t> tile_hdr, blk_part, obs_rec;
  DBuf<unsigned char> slots;
  DBuf<double> partial;
  int ntiles = 0;
  void upload(const TileSet& t, cudaStream_t st) {
    // an empty table goes up as 4 zeros (the slots as 16 zero bytes)
    auto up = [&](DBuf<uint32_t>& b, const auto& v) { upload_padded(b, v, v.empty() ? 4 : 0, st); };
    up(tile_hdr, t.tile_hdr);
    up(blk_part, t.blk_part);
    up(obs_rec, t.obs_rec);
    upload_padded(slots, t.slots, 16, st);
    partial.alloc(std::max<size_t>(1, t.blk_part.empty() ? 1 : t.blk_part.back()), st);
    ntiles = (int)(t.tile_hdr.size() / 4);
  }
  int prefetch_ahead = 0;
  MvTiles view(const int* blk_dim, const int* blk_off, int nblocks) const {
    MvTiles m;
    m.prefetch_ahead = prefetch_ahead;
    m.ntiles = ntiles;
    m.tile_hdr = reinterpret_cast<const uint4*>(tile_hdr.p);
    m.slots = slots.p;
    m.nblocks = nblocks;
    m.blk_dim = blk_dim;
    m.blk_off = blk_off;
    m.blk_part = blk_part.p;
    return m;
  }
};

// Auto operator switch: a PCG run of at least this many products moves the rest of the solve to the
// explicit S. One build of the rows costs about as much as this many tile products on the survey
// grids (plane500: ~2 ms of rows against ~60 us per product, the explicit product ~25 us).
constexpr uint64_t kExplicitSwitchTerms = 64;

template <typename T>
struct Solver {
  Context* ctx;
  cudaStream_t st;
  const NativeProblem& n;
  LmOptions opt;
  Layout L;
  Setup S;
  int N, P, D, nb, ng;
  bool direct;
  // device data
  DBuf<uint32_t> d_pt_off, d_obs_cam, d_obs_model, d_cam_group;
  DBuf<double> d_obs_px;
  DBuf<FixedCameraDev> d_models;
  DBuf<int> d_pose_off, d_pose_dim, d_intr_off, d_intr_dim;
  DBuf<uint8_t> d_pose_mask;
  DBuf<double> d_obs_bearing;
  DBuf<uint8_t> d_fixed_points;
  DBuf<double> d_pose[2], d_points[2], d_groups[2];
  int cur = 0;
  DBuf<T> d_rec;
  DBuf<float> d_rec32;
  TileSet T64, T32;
  TileSetDev dT64, dT32;
  bool mixed = false;
  DBuf<double> d_rw, d_vinv, d_vfac, d_ig, d_gp, d_ddiag;
  DBuf<PointSummary> d_summary, d_summary_part;
  DBuf<int> d_blk_off, d_blk_dim, d_blk_col, d_blk_edge, d_chunk_block, d_chunk_col, d_blk_chunk_begin, d_blk_chunk_end;
  DBuf<uint32_t> d_ent, d_ent_point, d_chunk_begin, d_chunk_end;
  DBuf<int> d_seg_col;
  DBuf<double> d_blk_out;
  DBuf<double> d_gfull, d_gred, d_diag, d_diag_minmax;
  DBuf<int> d_clamp;
  // pairs
  DBuf<int> d_xgrp_row, d_xgrp_col, d_blk_cross_begin, d_blk_cross_end;
  DBuf<uint32_t> d_xgrp_begin, d_xgrp_end, d_xpair_a, d_xpair_b, d_xpair_p;
  DBuf<double> d_xpair_out;
  DBuf<int> d_status;
  // explicit S: block rows, permutation and the banded tiled factor
  DBuf<uint32_t> d_blk_ent, d_nbr_begin;
  DBuf<int> d_ent_block, d_nbr, d_nbr_row, d_perm_off, d_perm_to_orig;
  DBuf<uint64_t> d_slot_off;
  DBuf<double> d_rows, d_tiles, d_winv, d_ztiles, d_perm_vec, d_marg_out, d_power;
  bool rows_valid = false;  // the rows hold S of the current assembly
  bool rows_attr = false;   // k_block_rows may take kRowSmemDoubles of dynamic shared memory
  bool asm_attr = false;    // k_block_tiles stages kAsmComp (TILE + 1) doubles in dynamic shared memory
  DBuf<double> d_asm_rec;   // per (block, segment) assembly records, kAsmRecordScale per partial element
  // PCG vectors
  DBuf<double> d_step, d_r, d_z, d_dir, d_q, d_factor, d_tmp, d_rhs, d_r64, d_e, d_dq, d_rr_part, d_rz_part;
  DBuf<int> d_fail;


  DBuf<double> d_scalars, d_cam_norm, d_ctl;
  DBuf<RedVec<4>> d_cand, d_cand_part;
  DBuf<RedVec<3>> d_met, d_met_part;
  DBuf<RedVec<1>> d_one, d_one_part;
  DBuf<RedVec<1>> d_norm_part;
  int red_blocks;
  uint64_t workspace_bytes = 0;
  bool explicit_op = false;

  Solver(Context* c, const NativeProblem& prob, const LmOptions& o)
      : ctx(c), st(o.stream ? static_cast<cudaStream_t>(o.stream) : c->stream), n(prob), opt(o) {
    L = make_layout(n);
    N = (int)n.obs_cam.size();
    P = (int)(n.points.size() / 3);
    D = L.D;
    ng = n.self_cal ? (int)n.group_dim.size() : 0;
    const double t0 = now();
    build_tables(n, L, S);
    build_explicit(n, L, S);
    if (opt.linear_solver == 0) {  // Auto: the budget's choice
      uint64_t nnz = 0, rows = 0, de = 0, ce = 0;
      pattern_counts(n, L, S, &nnz, &rows);
      opt.iterative = !auto_prefers_direct(n.self_cal, (uint64_t)N, D, (uint64_t)P, nnz, rows, opt.workspace_budget,
                                           &de, &ce);
      // a translation-only solve resolves Auto to the direct solver, so its final rank is exact
      // (native/mod.rs:398-407)
      if (!n.self_cal && !n.angular && n.translation_only) opt.iterative = false;
    }
    direct = !opt.iterative;
    // the PCG operator: the explicit S by block rows (rebuilt every assembly, a block-sparse product
    // that stays in L2) or the matrix-free tile product over the Jacobian records
    explicit_op = !direct && opt.matvec == 1;  // Auto starts matrix-free (see kExplicitSwitchTerms)
    const uint64_t bytes_before = tl_device_bytes;
    const double t1 = now();
    // mixed precision keeps only FP32 Jacobian records (and their tiles); FP64 mode only FP64 ones
    mixed = opt.precision == 1 && !direct;
    if (mixed)
      build_tiles(n, L, S, mv_tile_obs<float>(), T32);
    else
      build_tiles(n, L, S, mv_tile_obs<double>(), T64);
    const double t2 = now();
    nb = (int)S.blk_off.size();
    red_blocks = std::min(1024, grid_for(std::max(P, N), kReduceThreads));
    upload();
    sync();
    // the workspace: everything uploaded and allocated for the solve, and the banded factor of the
    // certificate (twice for self-calibration: the selected inverse has the factor's shape)
    workspace_bytes = (tl_device_bytes - bytes_before) +
                      sizeof(double) * (uint64_t)S.nt * kCTT * ((uint64_t)(S.bwt + 1) * (n.self_cal ? 2 : 1) + 1);
    if (opt.workspace_budget && workspace_bytes > opt.workspace_budget)
      throw SolveFailure{3, "GPU workspace " + std::to_string(workspace_bytes) + " bytes exceeds the workspace budget " +
                                std::to_string(opt.workspace_budget)};
    if (std::getenv("OMVGBA_PHASE_TIMES"))
      std::fprintf(stderr, "[omvgba] setup: tables %.3fs tiles %.3fs upload %.3fs\n", t1 - t0, t2 - t1, now() - t2);
  }

  DevView view() const {
    DevView v;
    v.P = P;
    v.ncam = n.ncam;
    v.self_cal = n.self_cal ? 1 : 0;
    v.pixel_model = n.pixel_model ? 1 : 0;
    v.pt_off = d_pt_off.p;
    v.obs_cam = d_obs_cam.p;
    v.obs_px = d_obs_px.p;
    v.obs_model = d_obs_model.p;
    v.models = d_models.p;
    v.cam_group = d_cam_group.p;
    v.pose_off = d_pose_off.p;
    v.pose_dim = d_pose_dim.p;
    v.pose_mask = d_pose_mask.p;
    v.angular = n.angular ? 1 : 0;
    v.obs_bearing = d_obs_bearing.p;
    v.intr_off = d_intr_off.p;
    v.intr_dim = d_intr_dim.p;
    v.fixed_points = d_fixed_points.p;
    return v;
  }
  DevState state(int which) const { return {d_pose[which].p, d_points[which].p, d_groups[which].p}; }
  // the FP32 records of mixed precision (assembly, pairs and candidate read them, computing in FP64)
  LinOut<float> lin32() const {
    return {d_rec32.p, dT32.obs_rec.p, mv_tile_obs<float>(), nullptr, nullptr, 0, d_rw.p, d_vinv.p, d_vfac.p, d_ig.p,
            d_gp.p, d_ddiag.p, d_summary.p, nullptr};
  }
  LinOut<T> lin() const {
    return {d_rec.p, dT64.obs_rec.p, mv_tile_obs<T>(), nullptr, nullptr, 0, d_rw.p, d_vinv.p, d_vfac.p, d_ig.p,
            d_gp.p, d_ddiag.p, d_summary.p, nullptr};
  }
  BlockTables tables() const {
    BlockTables b;
    b.nblocks = nb;
    b.blk_off = d_blk_off.p;
    b.blk_dim = d_blk_dim.p;
    b.blk_col = d_blk_col.p;
    b.blk_edge = d_blk_edge.p;
    b.ent = d_ent.p;
    b.ent_point = d_ent_point.p;
    b.nchunks = (int)S.chunk_block.size();
    b.chunk_block = d_chunk_block.p;
    b.chunk_col = d_chunk_col.p;
    b.chunk_begin = d_chunk_begin.p;
    b.chunk_end = d_chunk_end.p;
    b.blk_chunk_begin = d_blk_chunk_begin.p;
    b.blk_chunk_end = d_blk_chunk_end.p;
    return b;
  }
  // cross same-block pairs of the block-Jacobi preconditioner
  PairTables pairs() const {
    PairTables t;
    t.ngroups = (int)S.xgrp_row.size();
    t.grp_row = d_xgrp_row.p;
    t.grp_col = d_xgrp_col.p;
    t.grp_begin = d_xgrp_begin.p;
    t.grp_end = d_xgrp_end.p;
    t.pair_a = d_xpair_a.p;
    t.pair_b = d_xpair_b.p;
    t.pair_p = d_xpair_p.p;
    return t;
  }
  RowTables row_tables() const {
    RowTables r;
    r.nblocks = nb;
    r.blk_dim = d_blk_dim.p;
    r.blk_off = d_blk_off.p;
    r.blk_ent = d_blk_ent.p;
    r.ent = d_ent.p;
    r.ent_point = d_ent_point.p;
    r.seg_col = d_seg_col.p;
    r.ent_block = d_ent_block.p;
    r.pt_off = d_pt_off.p;
    r.nbr_begin = d_nbr_begin.p;
    r.nbr = d_nbr.p;
    r.nbr_row = d_nbr_row.p;
    r.slot_off = d_slot_off.p;
    r.entries = (uint32_t)S.nbr.size();
    return r;
  }
  TileBand tile_band() const { return TileBand{D, S.nt, S.bwt, d_tiles.p, d_winv.p}; }

  void upload() {
    std::vector<uint32_t> pt_off(n.pt_off.begin(), n.pt_off.end());
    d_pt_off.upload(pt_off.data(), pt_off.size(), st);
    d_obs_cam.upload(n.obs_cam.data(), n.obs_cam.size(), st);
    d_obs_px.upload(n.obs_px.data(), n.obs_px.size(), st);
    if (n.angular) d_obs_bearing.upload(n.obs_bearing.data(), n.obs_bearing.size(), st);
    upload_padded(d_obs_model, n.obs_model, 1, st);
    std::vector<FixedCameraDev> models = n.models;
    if (models.empty()) models.resize(1);
    d_models.upload(models.data(), models.size(), st);
    std::vector<uint32_t> cg = n.cam_group;
    if (cg.empty()) cg.assign(n.ncam, 0);
    d_cam_group.upload(cg.data(), cg.size(), st);
    d_pose_off.upload(L.pose_off.data(), L.pose_off.size(), st);
    d_pose_dim.upload(L.pose_dim.data(), L.pose_dim.size(), st);
    {
      std::vector<uint8_t> masks(std::max(n.ncam, 1), (uint8_t)3);
      if (n.explicit_masks)
        for (int c = 0; c < n.ncam; ++c) masks[c] = n.pose_mask[c];
      d_pose_mask.upload(masks.data(), masks.size(), st);
    }
    d_intr_off.upload(L.intr_off.data(), L.intr_off.size(), st);
    d_intr_dim.upload(L.intr_dim.data(), L.intr_dim.size(), st);
    d_fixed_points.upload(n.fixed_points.data(), n.fixed_points.size(), st);
    std::vector<double> pose(12 * (size_t)n.ncam);
    for (int c = 0; c < n.ncam; ++c) {
      for (int k = 0; k < 9; ++k) pose[12 * c + k] = n.rotation[9 * c + k];
      for (int k = 0; k < 3; ++k) pose[12 * c + 9 + k] = n.translation[3 * c + k];
    }
    for (int w = 0; w < 2; ++w) {
      d_pose[w].upload(pose.data(), pose.size(), st);
      d_points[w].upload(n.points.data(), n.points.size(), st);
      std::vector<double> gr = n.groups;
      if (gr.empty()) gr.assign(3, 0.0);
      d_groups[w].upload(gr.data(), gr.size(), st);
    }
    {
      if (!mixed) {
        dT64.upload(T64, st);
        d_rec.alloc((size_t)std::max(1, dT64.ntiles) * T64.tile * kRec, st);
        d_rec.zero();  // padding slots of partial tiles stay zero
      } else {
        dT32.upload(T32, st);
        d_rec32.alloc((size_t)std::max(1, dT32.ntiles) * T32.tile * kRec, st);
        d_rec32.zero();
      }
    }
    d_rw.alloc((size_t)2 * N, st);
    d_vinv.alloc((size_t)6 * P, st);
    d_vfac.alloc((size_t)6 * P, st);
    d_ig.alloc((size_t)3 * P, st);
    d_gp.alloc((size_t)3 * P, st);
    d_ddiag.alloc((size_t)3 * P, st);
    d_ddiag.zero();
    d_summary.alloc(P, st);
    d_summary_part.alloc(red_blocks, st);
    auto up_i = [&](DBuf<int>& b, const auto& v) { upload_padded(b, v, 1, st); };
    auto up_u = [&](DBuf<uint32_t>& b, const auto& v) { upload_padded(b, v, 1, st); };
    up_i(d_blk_off, S.blk_off);
    up_i(d_blk_dim, S.blk_dim);
    std::vector<int> col = S.blk_col;
    for (auto& c : col) c = std::max(c, 0);
    up_i(d_blk_col, col);
    up_i(d_blk_edge, S.blk_edge);
    up_u(d_ent, S.ent);
    up_u(d_ent_point, S.ent_point);
    up_i(d_chunk_block, S.chunk_block);
    up_i(d_chunk_col, S.chunk_col);
    up_u(d_chunk_begin, S.chunk_begin);
    up_u(d_chunk_end, S.chunk_end);
    up_i(d_blk_chunk_begin, S.blk_chunk_begin);
    up_i(d_blk_chunk_end, S.blk_chunk_end);
    up_i(d_seg_col, S.seg_col);
    up_i(d_xgrp_row, S.xgrp_row);
    up_i(d_xgrp_col, S.xgrp_col);
    up_u(d_xgrp_begin, S.xgrp_begin);
    up_u(d_xgrp_end, S.xgrp_end);
    up_u(d_xpair_a, S.xpair_a);
    up_u(d_xpair_b, S.xpair_b);
    up_u(d_xpair_p, S.xpair_p);
    up_i(d_blk_cross_begin, S.blk_cross_begin);
    up_i(d_blk_cross_end, S.blk_cross_end);
    d_blk_out.alloc((size_t)kAsmRec * std::max(1, nb), st);
    d_gfull.alloc(std::max(1, D), st);
    d_gred.alloc(std::max(1, D), st);
    d_diag.alloc(std::max(1, D), st);
    d_diag_minmax.alloc(2 * std::max(1, nb), st);
    d_clamp.alloc(std::max(1, nb), st);
    d_xpair_out.alloc((size_t)36 * std::max<size_t>(1, S.xgrp_row.size()), st);
    d_status.alloc(4, st);
    up_u(d_blk_ent, S.blk_ent);
    up_i(d_ent_block, S.ent_block);
    up_u(d_nbr_begin, S.nbr_begin);
    up_i(d_nbr, S.nbr);
    up_i(d_nbr_row, S.nbr_row);
    upload_padded(d_slot_off, S.slot_off, 1, st);
    up_i(d_perm_off, S.perm_off);
    up_i(d_perm_to_orig, S.perm_to_orig);
    d_rows.alloc(std::max<uint64_t>(1, S.slot_off.empty() ? 1 : S.slot_off.back()), st);
    d_perm_vec.alloc(std::max(1, D), st);
    d_power.alloc(2 * (size_t)std::max(1, D) + 2, st);
    for (DBuf<double>* b : {&d_step, &d_r, &d_z, &d_dir, &d_q, &d_tmp, &d_rhs, &d_r64, &d_e}) b->alloc(std::max(1, D), st);
    d_factor.alloc((size_t)42 * std::max(1, nb), st);
    d_dq.alloc(std::max(1, nb), st);
    d_rr_part.alloc(std::max(1, grid_for(nb, kUpdThreads)), st);
    d_rz_part.alloc(std::max(1, grid_for(nb, kUpdThreads)), st);
    d_fail.alloc(std::max(1, nb), st);
    {
      // one resident wave of product CTAs: how far ahead each CTA prefetches into L2
      int sms = 148, per64 = 1, per32 = 1;
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
      CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per64, k_mv_tiles<T, T>, mv_tile_obs<T>(), 0));
      CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per32, k_mv_tiles<float, float>, mv_tile_obs<float>(), 0));
      dT64.prefetch_ahead = per64 * sms;
      dT32.prefetch_ahead = per32 * sms;
    }
    d_scalars.alloc(16, st);
    d_ctl.alloc((sizeof(PcgCtl) + sizeof(double) - 1) / sizeof(double), st);
    d_cam_norm.alloc(std::max(1, n.ncam), st);
    d_cand.alloc(P, st);
    d_cand_part.alloc(red_blocks, st);
    d_met.alloc(P, st);
    d_met_part.alloc(red_blocks, st);
    d_one.alloc(std::max(N, n.ncam), st);
    d_one_part.alloc(red_blocks, st);
  }

  void sync() { CUDA_OK(cudaStreamSynchronize(st)); }
  void check_launch() { CUDA_OK(cudaGetLastError()); }

  template <int NV>
  RedVec<NV> reduce(const RedVec<NV>* in, int count, DBuf<RedVec<NV>>& part) {
    OMVGBA_LAUNCH(k_reduce_vec<NV>, red_blocks, kReduceThreads, 0, st, in, count, part.p);
    OMVGBA_LAUNCH(k_reduce_vec<NV>, 1, kReduceThreads, 0, st, part.p, red_blocks, part.p + 0);
    check_launch();
    RedVec<NV> h;
    CUDA_OK(copy_async(&h, part.p, sizeof(h), cudaMemcpyDeviceToHost, st));
    sync();
    return h;
  }

  Gauge gauge_for(int which, double scene) {
    Gauge g{};
    g.fixed_cam = n.gauge_cam;
    g.scene = scene;
    if (n.gauge_cam >= 0) {
      double t[3];
      CUDA_OK(copy_async(t, d_pose[which].p + 12 * n.gauge_cam + 9, sizeof(t), cudaMemcpyDeviceToHost, st));
      sync();
      g.baseline = std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
      for (int k = 0; k < 3; ++k) g.dir[k] = t[k] / g.baseline;
      // s2_tangent_basis (numerics/manifold.rs:118-131)
      double nv = std::sqrt(g.dir[0] * g.dir[0] + g.dir[1] * g.dir[1] + g.dir[2] * g.dir[2]);
      double tv[3] = {g.dir[0] / nv, g.dir[1] / nv, g.dir[2] / nv};
      double ref[3] = {0, 0, 0};
      if (std::fabs(tv[0]) <= std::fabs(tv[1]) && std::fabs(tv[0]) <= std::fabs(tv[2]))
        ref[0] = 1;
      else if (std::fabs(tv[1]) <= std::fabs(tv[2]))
        ref[1] = 1;
      else
        ref[2] = 1;
      auto cross = [](const double* a, const double* b, double* c) {
        c[0] = a[1] * b[2] - a[2] * b[1];
        c[1] = a[2] * b[0] - a[0] * b[2];
        c[2] = a[0] * b[1] - a[1] * b[0];
      };
      double b0[3], b1[3];
      cross(tv, ref, b0);
      double n0 = std::sqrt(b0[0] * b0[0] + b0[1] * b0[1] + b0[2] * b0[2]);
      for (int k = 0; k < 3; ++k) b0[k] /= n0;
      cross(tv, b0, b1);
      double n1 = std::sqrt(b1[0] * b1[0] + b1[1] * b1[1] + b1[2] * b1[2]);
      for (int k = 0; k < 3; ++k) {
        g.b0[k] = b0[k];
        g.b1[k] = b1[k] / n1;
      }
    }
    return g;
  }

  struct Assembly {
    bool valid;
    double cost, sq, point_red, grad_norm, min_rcond;
    uint64_t weak;
    double min_diag, max_diag;
    int clamp;
  };

  // Full linearization + camera-side reductions at the given damping.
  Assembly assemble(int which, const Gauge& g, const LossDev& loss, double lambda, bool build_rows) {
    DevView v = view();
    {
      const TileSetDev& ts = mixed ? dT32 : dT64;
      const MvTiles mt = ts.view(d_blk_dim.p, d_blk_off.p, nb);
      if (mt.ntiles > 0) {
        if (mixed)
          OMVGBA_LAUNCH(k_linearize_tiles<float>, mt.ntiles, mv_tile_obs<float>(), 0, st, v, state(which), g, loss,
                        lambda, lin32(), mt);
        else
          OMVGBA_LAUNCH(k_linearize_tiles<T>, mt.ntiles, mv_tile_obs<T>(), 0, st, v, state(which), g, loss, lambda,
                        lin(), mt);
      }
    }
    check_launch();
    OMVGBA_LAUNCH(k_reduce_summary, red_blocks, kReduceThreads, 0, st, d_summary.p, P, d_summary_part.p);
    OMVGBA_LAUNCH(k_reduce_summary, 1, kReduceThreads, 0, st, d_summary_part.p, red_blocks, d_summary_part.p);
    check_launch();
    BlockTables bt = tables();
    if (bt.nchunks > 0) {
      camera_sums();
      CUDA_OK(cudaMemsetAsync(d_gfull.p, 0, sizeof(double) * std::max(1, D), st));
      CUDA_OK(cudaMemsetAsync(d_gred.p, 0, sizeof(double) * std::max(1, D), st));
      CUDA_OK(cudaMemsetAsync(d_diag.p, 0, sizeof(double) * std::max(1, D), st));
      OMVGBA_LAUNCH(k_block_vectors, grid_for(nb, 64), 64, 0, st, bt, d_blk_out.p, d_gfull.p, d_gred.p, d_diag.p, d_clamp.p,
                                                     d_diag_minmax.p);
      check_launch();
    }
    rows_valid = false;
    if (build_rows && D > 0) this->build_rows();
    PointSummary ps;
    CUDA_OK(copy_async(&ps, d_summary_part.p, sizeof(ps), cudaMemcpyDeviceToHost, st));
    std::vector<double> mm(2 * std::max(nb, 1));
    std::vector<int> cl(std::max(nb, 1));
    std::vector<double> gvals(std::max(D, 1)), dvals(std::max(D, 1));
    if (nb > 0) {
      CUDA_OK(copy_async(mm.data(), d_diag_minmax.p, sizeof(double) * 2 * nb, cudaMemcpyDeviceToHost, st));
      CUDA_OK(copy_async(cl.data(), d_clamp.p, sizeof(int) * nb, cudaMemcpyDeviceToHost, st));
    }
    if (D > 0) {
      CUDA_OK(copy_async(gvals.data(), d_gfull.p, sizeof(double) * D, cudaMemcpyDeviceToHost, st));
      CUDA_OK(copy_async(dvals.data(), d_diag.p, sizeof(double) * D, cudaMemcpyDeviceToHost, st));
    }
    std::vector<double> gr(std::max(D, 1));
    if (D > 0) CUDA_OK(copy_async(gr.data(), d_gred.p, sizeof(double) * D, cudaMemcpyDeviceToHost, st));
    sync();
    Assembly a;
    a.valid = ps.invalid == 0.0;
    a.cost = ps.cost;
    a.sq = ps.sq;
    a.point_red = ps.point_red;
    a.grad_norm = ps.grad_norm;
    a.min_rcond = ps.min_rcond;
    a.weak = (uint64_t)ps.weak;
    double mn = INFINITY, mx = 0.0;
    a.clamp = 0;
    for (int b = 0; b < nb; ++b) {
      mn = std::min(mn, mm[2 * b]);
      mx = std::max(mx, mm[2 * b + 1]);
      a.clamp += cl[b];
    }
    a.min_diag = D == 0 ? 0.0 : mn;
    a.max_diag = mx;
    // scaled_gradient_inf_norm_prepared over the unreduced camera gradient (schur/assembly.rs:1092-1107)
    double gn = 0.0;
    bool finite = true;
    for (int i = 0; i < D; ++i) {
      double cv = dvals[i], val = gvals[i];
      double t = (std::isfinite(cv) && cv > 0.0) ? std::fabs(val) / std::sqrt(cv) : (val == 0.0 ? 0.0 : INFINITY);
      gn = std::max(gn, t);
      finite = finite && std::isfinite(gr[i]);
    }
    a.grad_norm = std::max(a.grad_norm, gn);
    a.valid = a.valid && finite && std::isfinite(a.cost);
    return a;
  }

  // ---- camera step ----
  bool direct_step(double lambda) {
    if (!factor_band(lambda, nullptr, 0.0)) return false;
    OMVGBA_LAUNCH(k_perm_gather, grid_for(D, 256), 256, 0, st, D, d_perm_to_orig.p, d_gred.p, -1.0, d_perm_vec.p);
    OMVGBA_LAUNCH(k_tile_solve, 1, 256, 0, st, tile_band(), d_perm_vec.p, d_status.p);
    OMVGBA_LAUNCH(k_perm_scatter, grid_for(D, 256), 256, 0, st, D, d_perm_to_orig.p, d_perm_vec.p, d_step.p);
    check_launch();
    return true;
  }

  // S of the current linearization (no damping) by block rows, from the FP64 or FP32 records.
  // The camera-side sums of the current linearization into the block assembly records (d_blk_out):
  // a pass over the record tiles, then each block's records in tile order.
  void camera_sums() {
    const int nb = (int)S.blk_off.size();
    BlockTables bt = tables();
    const TileSetDev& ts = mixed ? dT32 : dT64;
    MvTiles mt = ts.view(d_blk_dim.p, d_blk_off.p, nb);
    if (d_asm_rec.n != (size_t)kAsmRecordScale * ts.partial.n) {
      d_asm_rec.alloc((size_t)kAsmRecordScale * ts.partial.n, st);
      d_asm_rec.zero();  // record entries past a block's columns stay zero
    }
    if (!asm_attr) {
      CUDA_OK(cudaFuncSetAttribute(k_block_tiles<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)asm_smem_bytes<float>()));
      CUDA_OK(cudaFuncSetAttribute(k_block_tiles<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)asm_smem_bytes<T>()));
      asm_attr = true;
    }
    const uint32_t* pt_off = view().pt_off;
    if (mt.ntiles > 0) {
      if (mixed)
        OMVGBA_LAUNCH(k_block_tiles<float>, mt.ntiles, mv_tile_obs<float>(),
                      asm_smem_bytes<float>(), st, mt, lin32(), pt_off, d_asm_rec.p);
      else
        OMVGBA_LAUNCH(k_block_tiles<T>, mt.ntiles, mv_tile_obs<T>(),
                      asm_smem_bytes<T>(), st, mt, lin(), pt_off, d_asm_rec.p);
    }
    OMVGBA_LAUNCH(k_block_records, nb, 128, 0, st, mt, bt.blk_edge, d_asm_rec.p, d_blk_out.p);
  }

  void build_rows() {
    const int row_smem = (int)std::min<uint64_t>(S.max_row, (uint64_t)kRowSmemDoubles);
    const size_t smem = (size_t)row_smem * sizeof(double);
    if (!rows_attr) {
      CUDA_OK(cudaFuncSetAttribute(k_block_rows<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   kRowSmemDoubles * (int)sizeof(double)));
      CUDA_OK(cudaFuncSetAttribute(k_block_rows<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   kRowSmemDoubles * (int)sizeof(double)));
      rows_attr = true;
    }
    const bool timing = std::getenv("OMVGBA_PHASE_TIMES") != nullptr;
    if (timing) sync();
    const double t0 = now();
    if (mixed)
      OMVGBA_LAUNCH(k_block_rows<float>, nb, kRowThreads, smem, st, row_tables(), lin32(), row_smem, d_rows.p);
    else
      OMVGBA_LAUNCH(k_block_rows<T>, nb, kRowThreads, smem, st, row_tables(), lin(), row_smem, d_rows.p);
    check_launch();
    if (timing) {
      sync();
      std::fprintf(stderr, "[omvgba] block rows %.4fs (%d blocks, %zu entries)\n", now() - t0, nb, S.nbr.size());
    }
    rows_valid = true;
  }

  // y = (S + lambda diag) x from the rows
  void rows_matvec(const double* x, double* y, double lambda) {
    OMVGBA_LAUNCH(k_rows_matvec, grid_for((size_t)nb * 32, 256), 256, 0, st, row_tables(), d_rows.p, d_diag.p, lambda,
                  (const double*)nullptr, x, y, (double*)nullptr, (const PcgCtl*)nullptr);
    check_launch();
  }

  // Cholesky of (S + lambda diag) -- equilibrated as scale S scale and shifted by -shift I when scale
  // is given -- into the banded tiles; true when every pivot is finite and positive.
  static constexpr size_t kMaxTileBytes = size_t(16) << 30;
  static constexpr int kGraphColumns = 64;  // tile columns from which a column loop runs as a graph
  // Runs a long fixed sequence of launches (a tile-column loop) as one CUDA graph: captured on the
  // solver's stream, instantiated, launched and waited for, so the device runs the columns back to
  // back whatever the host is doing meanwhile.
  template <typename Body>
  void run_as_graph(Body body) {
    if (S.nt < kGraphColumns) {  // short loops: capture and instantiation would cost more than they save
      body();
      return;
    }
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    CUDA_OK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    body();
    const cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (ce != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      CUDA_OK(ce);
    }
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    CUDA_OK(ie);
    const cudaError_t le = cudaGraphLaunch(exec, st);
    const cudaError_t se = cudaStreamSynchronize(st);
    cudaGraphExecDestroy(exec);
    CUDA_OK(le);
    CUDA_OK(se);
  }

  bool factor_band(double lambda, const double* scale, double shift) {
    if (D == 0) return true;
    const double t_factor = now();
    const size_t count = (size_t)S.nt * (S.bwt + 1) * kCTT;
    if (sizeof(double) * count > kMaxTileBytes)
      throw SolveFailure{3, "the banded factor of the reduced camera system exceeds 16 GiB"};
    if (d_tiles.n != count) d_tiles.alloc(count, st);
    if (d_winv.n != (size_t)S.nt * kCTT) d_winv.alloc((size_t)S.nt * kCTT, st);
    // per device and cheap: set on every factorization
    CUDA_OK(cudaFuncSetAttribute(k_tile_trsm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsmSmem));
    CUDA_OK(cudaFuncSetAttribute(k_tile_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUpdateSmem));
    CUDA_OK(cudaMemsetAsync(d_tiles.p, 0, sizeof(double) * count, st));
    OMVGBA_LAUNCH(k_set_int, 1, 1, 0, st, d_status.p, 1);
    const TileBand tb = tile_band();
    OMVGBA_LAUNCH(k_rows_to_tiles, grid_for(S.nbr.size(), 128), 128, 0, st, row_tables(), d_rows.p, d_perm_off.p,
                  d_diag.p, lambda, scale, shift, tb);
    OMVGBA_LAUNCH(k_tiles_pad, 1, kCT, 0, st, tb);
    run_as_graph([&] {
      for (int k = 0; k < S.nt; ++k) {
        OMVGBA_LAUNCH(k_tile_potrf, 1, 256, 0, st, tb, k, d_status.p);
        const int m = std::min(S.bwt, S.nt - 1 - k);
        if (m > 0) {
          OMVGBA_LAUNCH(k_tile_trsm, m, 256, kTrsmSmem, st, tb, k, d_status.p);
          OMVGBA_LAUNCH(k_tile_update, m * (m + 1) / 2, 256, kUpdateSmem, st, tb, k, d_status.p);
        }
      }
    });
    check_launch();
    int ok = 0;
    CUDA_OK(copy_async(&ok, d_status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    sync();
    if (std::getenv("OMVGBA_PHASE_TIMES"))
      std::fprintf(stderr, "[omvgba] band factor %.4fs (nt %d bwt %d) ok %d\n", now() - t_factor, S.nt, S.bwt, ok);
    return ok != 0;
  }

  // Camera rank of the final undamped system (sparse/direct.rs:288-455; the native lowering fixes the
  // gauge with pose masks, so the expected nullity is zero): D <= dense_rank_limit: every eigenvalue
  // of the Jacobi-equilibrated S above tol = 64 eps D lambda_max, i.e. S_eq - tol I positive definite;
  // above the limit: S itself factors. Returns 0 (full rank) or 2 (rank deficient or indefinite);
  // *factored_s tells whether the band holds the factor of S itself.
  int rank_certificate(bool* factored_s) {
    *factored_s = false;
    if (D == 0) return 0;
    if (D > opt.dense_rank_limit) {
      const bool ok = factor_band(0.0, nullptr, 0.0);
      *factored_s = ok;
      return ok ? 0 : 2;
    }
    std::vector<double> dg(D);
    OMVGBA_LAUNCH(k_rows_diag, grid_for(nb, 128), 128, 0, st, row_tables(), d_rows.p, d_tmp.p);
    check_launch();
    CUDA_OK(copy_async(dg.data(), d_tmp.p, sizeof(double) * D, cudaMemcpyDeviceToHost, st));
    sync();
    double ds = 0.0;
    for (int i = 0; i < D; ++i) ds = std::max(ds, std::fabs(dg[i]));
    if (!(std::isfinite(ds) && ds > 0.0)) return 2;
    const double fl = 64.0 * kEps * ds;
    std::vector<double> sc(D);
    for (int i = 0; i < D; ++i) {
      if (!std::isfinite(dg[i])) return 2;
      sc[i] = 1.0 / std::sqrt(std::max(dg[i], fl));
    }
    CUDA_OK(copy_async(d_e.p, sc.data(), sizeof(double) * D, cudaMemcpyHostToDevice, st));
    OMVGBA_LAUNCH(k_power_iteration, 1, 1024, 0, st, row_tables(), d_rows.p, d_e.p, D, d_power.p, d_power.p + D,
                  d_power.p + 2 * (size_t)D);
    check_launch();
    double out[2];
    CUDA_OK(copy_async(out, d_power.p + 2 * (size_t)D, sizeof(out), cudaMemcpyDeviceToHost, st));
    sync();
    const double largest = std::fabs(out[0]);
    if (out[1] == 0.0 || !(std::isfinite(largest) && largest > 0.0)) return 2;
    const double tol = 64.0 * kEps * D * largest;
    if (std::getenv("OMVGBA_PHASE_TIMES"))
      std::fprintf(stderr, "[omvgba] rank: lambda_max %.6e tol %.3e\n", largest, tol);
    return factor_band(0.0, d_e.p, tol) ? 0 : 2;
  }

  // Marginal covariances (S^-1)_gg of the free intrinsic groups of the final undamped system
  // (sparse/covariance.rs:564-587 without the weight normalization): 9 values per group, row-major
  // (the dim x dim corner used). False when S does not factor.
  bool intrinsic_marginals(bool factored_s, std::vector<double>& out) {
    out.assign(9 * (size_t)std::max(ng, 1), 0.0);
    std::vector<int> pos, dims, gid;
    for (int g = 0; g < ng; ++g)
      if (L.intr_dim[g] > 0 && S.grp_block[g] >= 0) {
        const int b = S.grp_block[g];
        for (int k = 0; k < 3; ++k) pos.push_back(k < L.intr_dim[g] ? S.perm_off[b] + k : S.perm_off[b]);
        dims.push_back(L.intr_dim[g]);
        gid.push_back(g);
      }
    if (gid.empty()) return true;
    if (!factored_s && !factor_band(0.0, nullptr, 0.0)) return false;
    // selected inverse of S inside the band (Takahashi recurrence), last tile column first
    const size_t count = (size_t)S.nt * (S.bwt + 1) * kCTT;
    d_ztiles.alloc(count, st);
    CUDA_OK(cudaFuncSetAttribute(k_takahashi_partial, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTakahashiSmem));
    CUDA_OK(cudaFuncSetAttribute(k_takahashi_offdiag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTakahashiSmem));
    CUDA_OK(cudaFuncSetAttribute(k_takahashi_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTakahashiSmem));
    const TileBand tl = tile_band();
    const TileBand tz{D, S.nt, S.bwt, d_ztiles.p, nullptr};
    // scratch: the split partial sums of one column and the diagonal shares of its tiles
    const int max_split = (S.bwt + kTakahashiChunk - 1) / kTakahashiChunk;
    DBuf<double> d_zpart, d_zq;
    d_zpart.alloc((size_t)std::max(S.bwt, 1) * std::max(max_split, 1) * kCTT, st);
    d_zq.alloc((size_t)std::max(S.bwt, 1) * kCTT, st);
    run_as_graph([&] {
      for (int j = S.nt - 1; j >= 0; --j) {
        const int m = std::min(S.bwt, S.nt - 1 - j);
        if (m > 0) {
          const int nsplit = (m + kTakahashiChunk - 1) / kTakahashiChunk;
          OMVGBA_LAUNCH(k_takahashi_partial, dim3(m, nsplit), 256, kTakahashiSmem, st, tl, tz, j, d_zpart.p,
                        d_status.p);
          OMVGBA_LAUNCH(k_takahashi_offdiag, m, 256, kTakahashiSmem, st, tl, tz, j, nsplit, d_zpart.p, d_zq.p,
                        d_status.p);
        }
        OMVGBA_LAUNCH(k_takahashi_diag, 1, 256, kTakahashiSmem, st, tl, tz, j, m, d_zq.p, d_status.p);
      }
    });
    DBuf<int> d_pos, d_dims;
    d_pos.upload(pos.data(), pos.size(), st);
    d_dims.upload(dims.data(), dims.size(), st);
    const int total = (int)gid.size();
    d_marg_out.alloc(9 * (size_t)total, st);
    OMVGBA_LAUNCH(k_z_marginals, grid_for(total, 128), 128, 0, st, tz, total, d_pos.p, d_dims.p, d_marg_out.p,
                  d_status.p);
    check_launch();
    std::vector<double> m(9 * (size_t)total);
    int ok = 0;
    CUDA_OK(copy_async(m.data(), d_marg_out.p, sizeof(double) * m.size(), cudaMemcpyDeviceToHost, st));
    CUDA_OK(copy_async(&ok, d_status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    sync();
    d_ztiles.release();
    if (!ok) return false;
    for (int i = 0; i < total; ++i)
      for (int k = 0; k < 9; ++k) out[9 * (size_t)gid[i] + k] = m[9 * (size_t)i + k];
    return true;
  }

  void dots(std::initializer_list<std::pair<const double*, const double*>> pairs, double* out) {
    DotArgs a{};
    int k = 0;
    for (auto& pr : pairs) {
      a.a[k] = pr.first;
      a.b[k] = pr.second;
      ++k;
    }
    a.count = k;
    OMVGBA_LAUNCH(k_dots, 1, 1024, 0, st, a, D, d_scalars.p);
    check_launch();
    CUDA_OK(copy_async(out, d_scalars.p, sizeof(double) * k, cudaMemcpyDeviceToHost, st));
    sync();
  }

  // y = S_lambda x (implicit, matrix-free); ctl: optional PCG control for graph-launched iterations
  // fp32: use the FP32 record copy (mixed precision inner solves)
  int mv_finalize_ctas() const { return std::max(1, grid_for((size_t)nb * 32, 256)); }
  // xy: optional per-finalize-CTA sums of x_b . y_b over the CTA's blocks (the PCG curvature terms)
  // pdl_tiles / pdl: launch the tile pass / the finalize as programmatic dependents of the kernel
  // before them (inside the PCG graph)
  void matvec(const double* x, double* y, double lambda, const PcgCtl* ctl = nullptr, bool fp32 = false,
              double* xy = nullptr, bool pdl_tiles = false, bool pdl = false) {
    if (explicit_op) {  // block-sparse product of the explicit S (FP64 rows)
      launch_pdl(pdl_tiles, k_rows_matvec, mv_finalize_ctas(), 256, st, row_tables(), (const double*)d_rows.p,
                 (const double*)d_diag.p, lambda, (const double*)nullptr, x, y, xy, ctl);
      check_launch();
      return;
    }
    matvec_tiles(x, ctl, fp32, pdl_tiles);
    const TileSetDev& ts = mixed ? dT32 : dT64;
    MvTiles mt = ts.view(d_blk_dim.p, d_blk_off.p, nb);
    launch_pdl(pdl, k_mv_tiles_finalize, mv_finalize_ctas(), 256, st, mt, ts.partial.p, d_diag.p, lambda, x, y, xy,
               ctl);
    check_launch();
  }
  // The tile pass of the product alone: the per-(segment, parameter) partials.
  void matvec_tiles(const double* x, const PcgCtl* ctl, bool fp32, bool pdl = false) {
    const TileSetDev& ts = mixed ? dT32 : dT64;
    MvTiles mt = ts.view(d_blk_dim.p, d_blk_off.p, nb);
    if (mt.ntiles > 0) {
      if (fp32)
        launch_pdl(pdl, k_mv_tiles<float, float>, mt.ntiles, mv_tile_obs<float>(), st, mt, d_rec32.p, d_vfac.p, x,
                   ts.partial.p, ctl);
      else if (mixed)  // FP64 arithmetic on the FP32 records: the refinement's residual product
        launch_pdl(pdl, k_mv_tiles<float, double>, mt.ntiles, mv_tile_obs<float>(), st, mt, d_rec32.p, d_vfac.p, x,
                   ts.partial.p, ctl);
      else
        launch_pdl(pdl, k_mv_tiles<T, T>, mt.ntiles, mv_tile_obs<T>(), st, mt, d_rec.p, d_vfac.p, x, ts.partial.p,
                   ctl);
    }
  }

  bool factor_preconditioner(double lambda) {
    BlockTables bt = tables();
    PairTables xt = pairs();
    if (explicit_op) {
      OMVGBA_LAUNCH(k_block_factor_rows, grid_for(nb, 64), 64, 0, st, row_tables(), d_rows.p, d_diag.p, lambda,
                    d_factor.p, d_fail.p);
    } else if (xt.ngroups > 0) {
      if (mixed)
        OMVGBA_LAUNCH(k_pairs<float>, xt.ngroups, 32, 0, st, xt, bt, lin32(), d_seg_col.p, d_xpair_out.p);
      else
        OMVGBA_LAUNCH(k_pairs<T>, xt.ngroups, 32, 0, st, xt, bt, lin(), d_seg_col.p, d_xpair_out.p);
    }
    if (!explicit_op)
      OMVGBA_LAUNCH(k_block_factor, grid_for(nb, 64), 64, 0, st, bt, d_blk_out.p, d_diag.p, lambda, d_xpair_out.p,
                    d_blk_cross_begin.p, d_blk_cross_end.p, d_factor.p, d_fail.p);
    check_launch();
    std::vector<int> fail(std::max(nb, 1));
    if (nb > 0) CUDA_OK(copy_async(fail.data(), d_fail.p, sizeof(int) * nb, cudaMemcpyDeviceToHost, st));
    sync();
    for (int b = 0; b < nb; ++b)
      if (fail[b]) return false;
    return true;
  }
  void precond(const double* r, double* z, const PcgCtl* ctl = nullptr) {
    OMVGBA_LAUNCH(k_block_precond, grid_for(nb, 64), 64, 0, st, tables(), d_factor.p, r, z, ctl);
    check_launch();
  }

  struct PcgResult {
    bool accepted = false;
    bool exhausted = false;
    uint64_t terms = 0;
    double rel = NAN;
  };
  // pcg::solve (sparse/pcg.rs:23-119), require_bounded_residual, for S x = b with x0 = 0. The
  // iteration body runs as a CUDA graph; the host polls the device status every kPoll iterations.
  // confirm: when the recursive residual meets the tolerance, confirm it with the true residual
  // b - S x (the reference's rule); without it the recursive residual decides (inner solves of the
  // mixed-precision refinement, whose outer loop checks the FP64 residual). fp32: FP32 products.
  static constexpr int kPoll = 8;
  PcgResult pcg_run(const double* b, double* x, double lambda, uint64_t max_it, double tol, bool fp32, bool confirm) {
    double t_start = now();
    int launches = 0, restarts = 0;
    PcgResult res;
    double t_ready = 0.0;  // host clock when the graph is instantiated
    struct Report {
      double t0;
      const double* t_ready;
      int* launches;
      int* restarts;
      PcgResult* res;
      bool fp32;
      ~Report() {
        if (std::getenv("OMVGBA_PCG_TRACE"))
          std::fprintf(stderr, "[pcg%s] %.3f ms terms %llu accepted %d rel %.3e launches %d restarts %d setup %.3f ms\n",
                       fp32 ? "32" : "64", (now() - t0) * 1e3, (unsigned long long)res->terms, (int)res->accepted,
                       res->rel, *launches, *restarts, *t_ready > 0.0 ? (*t_ready - t0) * 1e3 : 0.0);
      }
    } rpt{t_start, &t_ready, &launches, &restarts, &res, fp32};
    CUDA_OK(cudaMemsetAsync(x, 0, sizeof(double) * D, st));
    CUDA_OK(copy_async(d_r.p, b, sizeof(double) * D, cudaMemcpyDeviceToDevice, st));
    double h[4];
    dots({{d_r.p, d_r.p}}, h);
    double n0 = std::sqrt(h[0]);
    if (!std::isfinite(n0)) return res;
    if (n0 == 0.0) {
      res.accepted = true;
      res.rel = 0.0;
      return res;
    }
    precond(d_r.p, d_z.p);
    CUDA_OK(copy_async(d_dir.p, d_z.p, sizeof(double) * D, cudaMemcpyDeviceToDevice, st));
    dots({{d_r.p, d_z.p}}, h);
    double rho = h[0];
    if (!(std::isfinite(rho) && rho > 0.0)) return res;
    if (max_it == 0) return res;
    PcgCtl ctl{};
    ctl.n0 = n0;
    ctl.rho_slot[0] = rho;
    ctl.tol = tol;
    ctl.status = kRunning;
    ctl.terms = 0;
    ctl.max_it = (int)std::min<uint64_t>(max_it, (uint64_t)INT32_MAX);
    PcgCtl* dctl = reinterpret_cast<PcgCtl*>(d_ctl.p);
    CUDA_OK(copy_async(dctl, &ctl, sizeof(ctl), cudaMemcpyHostToDevice, st));
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    const uint64_t launches_before = tl_telemetry.launches;
    CUDA_OK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    // one poll batch (kPoll iterations, an even count) per graph: even iterations read rho slot 0,
    // odd ones slot 1 (every kernel after the graph's first is a programmatic dependent of the one
    // before it)
    static_assert(kPoll % 2 == 0, "the rho slots alternate");
    for (int it = 0; it < kPoll; ++it) {
      const int slot = it & 1;
      matvec(d_dir.p, d_q.p, lambda, dctl, fp32, d_dq.p, it > 0, true);
      const int nupd = grid_for(nb, kUpdThreads);
      launch_pdl(true, k_pcg_update_precond, nupd, kUpdThreads, st, tables(), d_factor.p, d_dq.p, mv_finalize_ctas(),
                 d_dir.p, d_q.p, x, d_r.p, d_z.p, d_rr_part.p, d_rz_part.p, slot, dctl);
      launch_pdl(true, k_pcg_direction, grid_for(D, 256), 256, st, D, d_rr_part.p, d_rz_part.p, nupd, d_z.p, d_dir.p,
                 slot, dctl);
    }
    CUDA_OK(cudaStreamEndCapture(st, &graph));
    const uint64_t kernels_per_graph = tl_telemetry.launches - launches_before;  // counted at capture
    tl_telemetry.launches = launches_before;
    CUDA_OK(cudaGraphInstantiate(&exec, graph, 0));
    t_ready = now();
    struct GraphGuard {
      cudaGraph_t g;
      cudaGraphExec_t e;
      ~GraphGuard() {
        cudaGraphExecDestroy(e);
        cudaGraphDestroy(g);
      }
    } guard{graph, exec};
    auto recompute = [&]() {
      matvec(x, d_q.p, lambda, nullptr, fp32);
      OMVGBA_LAUNCH(k_sub, grid_for(D, 256), 256, 0, st, D, b, d_q.p, d_r.p);
      check_launch();
    };
    PcgCtl* mirror = static_cast<PcgCtl*>(tl_poll.get(2 * sizeof(PcgCtl)));
    if (!mirror) throw SolveFailure{8, "pinned host memory for the PCG status is not available"};
    struct Events {
      cudaEvent_t e[2] = {nullptr, nullptr};
      ~Events() {
        for (cudaEvent_t x : e)
          if (x) cudaEventDestroy(x);
      }
    } ev;
    for (cudaEvent_t& e : ev.e) CUDA_OK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    // one batch: kPoll iterations, then the status copied into mirror[i]
    auto enqueue = [&](int i) {
      CUDA_OK(cudaGraphLaunch(exec, st));  // kPoll iterations
      tl_telemetry.launches += kernels_per_graph;
      launches += kPoll;
      CUDA_OK(cudaMemcpyAsync(&mirror[i], dctl, sizeof(PcgCtl), cudaMemcpyDeviceToHost, st));
      tl_telemetry.d2h += sizeof(PcgCtl);
      CUDA_OK(cudaEventRecord(ev.e[i], st));
    };
    // The next batch is enqueued before the host waits for the current batch's status, so the device
    // keeps running while the host reads it. A batch that runs after the loop stopped changes nothing
    // the host reads: its products and updates return at once, and at the iteration limit its
    // direction kernels only rewrite the direction and the term count, which the host replaces. The
    // host waits for that batch before it acts on the status.
    int cur = 0;
    enqueue(cur);
    for (;;) {
      enqueue(cur ^ 1);
      CUDA_OK(cudaEventSynchronize(ev.e[cur]));
      ctl = mirror[cur];
      cur ^= 1;
      if (ctl.status == kRunning) continue;
      CUDA_OK(cudaEventSynchronize(ev.e[cur]));
      if (ctl.status == kRejected) {
        res.terms = ctl.terms;
        return res;
      }
      if (ctl.status == kExhausted) break;
      if (!confirm) {  // kCheckResidual without confirmation: the recursive residual decides
        res.accepted = true;
        res.terms = ctl.terms;
        res.rel = ctl.ratio;
        return res;
      }
      // kCheckResidual: the recursive residual met the tolerance; confirm with the true residual
      ++restarts;
      recompute();
      dots({{d_r.p, d_r.p}}, h);
      double tr = std::sqrt(h[0]) / n0;
      if (std::isfinite(tr) && tr <= tol) {
        res.accepted = true;
        res.terms = ctl.terms;
        res.rel = tr;
        return res;
      }
      if (!std::isfinite(tr)) {
        res.terms = ctl.terms;
        return res;
      }
      precond(d_r.p, d_z.p);
      CUDA_OK(copy_async(d_dir.p, d_z.p, sizeof(double) * D, cudaMemcpyDeviceToDevice, st));
      dots({{d_r.p, d_z.p}}, h);
      double nrho = h[0];
      if (!(std::isfinite(nrho) && nrho > 0.0)) {
        res.terms = ctl.terms;
        res.rel = tr;
        return res;
      }
      if ((uint64_t)ctl.terms >= max_it) break;
      ctl.rho_slot[0] = nrho;
      ctl.status = kRunning;
      CUDA_OK(copy_async(dctl, &ctl, sizeof(ctl), cudaMemcpyHostToDevice, st));
      enqueue(cur);
    }
    recompute();
    dots({{d_r.p, d_r.p}}, h);
    res.terms = max_it;
    res.rel = std::sqrt(h[0]) / n0;
    res.exhausted = true;
    return res;
  }

  PcgResult pcg(double lambda, uint64_t max_it, double tol) {
    OMVGBA_LAUNCH(k_neg_copy, grid_for(D, 256), 256, 0, st, D, d_gred.p, d_rhs.p);
    check_launch();
    return pcg_run(d_rhs.p, d_step.p, lambda, max_it, tol, false, true);
  }

  // Mixed precision: FP32-product PCG inner solves refined against the FP64 residual
  // r = -g - S x; the step is accepted when the FP64 relative residual meets the tolerance, the
  // same acceptance rule as the FP64 solve, within the same iteration budget.
  PcgResult pcg_mixed(double lambda, uint64_t max_it, double tol) {
    PcgResult res;
    OMVGBA_LAUNCH(k_neg_copy, grid_for(D, 256), 256, 0, st, D, d_gred.p, d_rhs.p);
    check_launch();
    double h[4];
    dots({{d_rhs.p, d_rhs.p}}, h);
    double n0 = std::sqrt(h[0]);
    if (!std::isfinite(n0)) return res;
    CUDA_OK(cudaMemsetAsync(d_step.p, 0, sizeof(double) * D, st));
    if (n0 == 0.0) {
      res.accepted = true;
      res.rel = 0.0;
      return res;
    }
    CUDA_OK(copy_async(d_r64.p, d_rhs.p, sizeof(double) * D, cudaMemcpyDeviceToDevice, st));
    double rel = 1.0;
    uint64_t terms = 0;
    for (int outer = 0; outer < 32 && terms < max_it; ++outer) {
      double eta = std::min(0.5, std::max(0.5 * tol / rel, 1e-4));
      PcgResult in = pcg_run(d_r64.p, d_e.p, lambda, max_it - terms, eta, true, false);
      terms += in.terms;
      if (!in.accepted && !in.exhausted) {
        res.terms = terms;
        return res;  // curvature or finiteness failure
      }
      OMVGBA_LAUNCH(k_axpy, grid_for(D, 256), 256, 0, st, D, 1.0, d_e.p, d_step.p);
      matvec(d_step.p, d_q.p, lambda, nullptr, false);
      OMVGBA_LAUNCH(k_sub, grid_for(D, 256), 256, 0, st, D, d_rhs.p, d_q.p, d_r64.p);
      check_launch();
      dots({{d_r64.p, d_r64.p}}, h);
      double nrel = std::sqrt(h[0]) / n0;
      if (!std::isfinite(nrel)) {
        res.terms = terms;
        return res;
      }
      if (nrel <= tol) {
        res.accepted = true;
        res.terms = terms;
        res.rel = nrel;
        return res;
      }
      if (nrel > 0.9 * rel) {  // the FP32 correction no longer reduces the FP64 residual
        res.terms = terms;
        res.rel = nrel;
        return res;
      }
      rel = nrel;
    }
    res.terms = terms;
    res.rel = rel;
    return res;
  }

  double scene_scale_host() {
    // observed_scene_scale (optimizer.rs:630-675) for calibrated, scene_scale (:620-628) for self-cal
    if (n.gauge_cam >= 0) {
      const double* t = &n.translation[3 * n.gauge_cam];
      return std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
    }
    if (n.self_cal) {
      double s = 0.0;
      for (size_t i = 0; i < n.points.size(); ++i) s += n.points[i] * n.points[i];
      return std::max(std::sqrt(s / double(P)), kMinPositive);
    }
    double scale = 0.0, sq = 1.0;
    size_t count = 0;
    for (int p = 0; p < P; ++p) {
      if (n.pt_off[p] == n.pt_off[p + 1]) continue;
      count++;
      for (int k = 0; k < 3; ++k) {
        double m = std::fabs(n.points[3 * p + k]);
        if (m == 0.0) continue;
        if (scale < m) {
          double r = scale / m;
          sq = 1.0 + sq * r * r;
          scale = m;
        } else {
          double r = m / scale;
          sq += r * r;
        }
      }
    }
    if (scale == 0.0 || count == 0) return kMinPositive;
    double rms = scale * std::sqrt(sq / double(count));
    return std::isfinite(rms) ? std::max(rms, kMinPositive) : scale;
  }

  void metrics(int which, const LossDev& loss, double* cost, double* rmse) {
    OMVGBA_LAUNCH(k_metrics, grid_for(P, 128), 128, 0, st, view(), state(which), loss, d_met.p);
    check_launch();
    RedVec<3> r = reduce<3>(d_met.p, P, d_met_part);
    if (r.v[2] > 0.0) {
      *cost = INFINITY;
      *rmse = INFINITY;
      return;
    }
    *cost = r.v[0];
    *rmse = std::sqrt(r.v[1] / double(2 * (size_t)N));
  }

  double t_assemble = 0, t_solve = 0, t_candidate = 0;
  static double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
  }

  // Resident use (one upload, many solves): the initial state is kept and restored before each solve.
  DBuf<double> d_pose_init, d_points_init, d_groups_init;
  void keep_initial() {
    for (auto pr : {std::make_pair(&d_pose_init, &d_pose[cur]), std::make_pair(&d_points_init, &d_points[cur]),
                    std::make_pair(&d_groups_init, &d_groups[cur])}) {
      pr.first->alloc(pr.second->n, st);
      CUDA_OK(copy_async(pr.first->p, pr.second->p, sizeof(double) * pr.second->n, cudaMemcpyDeviceToDevice, st));
    }
  }
  void restore_initial() {
    cur = 0;
    for (auto pr : {std::make_pair(&d_pose_init, &d_pose[0]), std::make_pair(&d_points_init, &d_points[0]),
                    std::make_pair(&d_groups_init, &d_groups[0])})
      CUDA_OK(copy_async(pr.second->p, pr.first->p, sizeof(double) * pr.first->n, cudaMemcpyDeviceToDevice, st));
    t_assemble = t_solve = t_candidate = 0;
  }

  NativeReport refine(std::vector<double>& rotation, std::vector<double>& translation, std::vector<double>& points,
                      std::vector<double>& groups) {
    NativeReport rep;
    double t_begin = now();
    double scene = scene_scale_host();
    // stages (continuation.rs:18-74)
    struct Stage {
      LossDev loss;
      uint64_t iters;
    } stages[3];
    const LossDev l2{kLossL2, 0.0};
    if (opt.loss.kind == kLossCauchy) {
      uint64_t w = std::min<uint64_t>(opt.max_iterations / 4, 5);
      stages[0] = {l2, w};
      stages[1] = {opt.loss, opt.max_iterations - w};
      stages[2] = {l2, 0};
    } else {
      stages[0] = {opt.loss, opt.max_iterations};
      stages[1] = {l2, 0};
      stages[2] = {l2, 0};
    }
    int target = 0;
    for (int i = 2; i >= 0; --i)
      if (stages[i].iters > 0) {
        target = i;
        break;
      }
    bool reuse = false;
    for (auto& s : stages)
      if (s.iters > 0) {
        reuse = s.loss.kind == opt.loss.kind && s.loss.scale == opt.loss.scale;
        break;
      }
    bool have_initial = false;
    double init_cost = INFINITY, init_rmse = INFINITY;
    if (!reuse) {
      metrics(cur, opt.loss, &init_cost, &init_rmse);
      have_initial = true;
    }
    // Nielsen controller (numerics/refine/nonlinear/controller.rs:6-91) and run state (run_state.rs)
    double lambda = direct ? 1e-4 : 1e-1, nu = 2.0;
    auto increase = [&]() {
      lambda = std::min(lambda * nu, 1e12);
      nu = std::min(nu * 2.0, 1e12);
    };
    uint64_t iterations = 0, accepted = 0, target_accepted = 0, rej[4] = {0, 0, 0, 0};
    int convergence = -1;
    uint64_t pcg_terms = 0;
    double iter_tol = std::min(std::sqrt(opt.relative_cost_tolerance), 1e-6);
    bool done = false;
    bool switch_pending = false;  // the Auto switch takes effect at the next assembly
    int cand = 1 - cur;
    size_t free_points = 0;
    for (int p = 0; p < P; ++p) free_points += n.fixed_points[p] ? 0 : 1;
    for (int si = 0; si < 3 && !done; ++si) {
      bool confirm = false;
      for (uint64_t it = 0; it < stages[si].iters; ++it) {
        iterations++;
        double t0 = now();
        if (switch_pending) {
          explicit_op = true;
          switch_pending = false;
        }
        Gauge g = gauge_for(cur, scene);
        Assembly a = assemble(cur, g, stages[si].loss, lambda, direct || explicit_op);
        double t1 = now();
        t_assemble += t1 - t0;
        if (!have_initial && std::isfinite(a.cost) && std::isfinite(a.sq) && N > 0) {
          init_cost = a.cost;
          init_rmse = std::sqrt(a.sq / double(2 * (size_t)N));
          have_initial = true;
        }
        if (!a.valid) {
          rej[0]++;
          increase();
          continue;
        }
        double current = a.cost;
        if (si == target && convergence < 0 && std::isfinite(a.grad_norm) && a.grad_norm >= 0.0 &&
            std::isfinite(current) && a.grad_norm <= opt.gradient_tolerance * (1.0 + std::fabs(current))) {
          convergence = 1;
          done = true;
          break;
        }
        bool iterative_step = false;
        double rel_res = 0.0;
        bool solved = true;
        if (direct) {
          solved = D == 0 || direct_step(lambda);
        } else {
          solved = factor_preconditioner(lambda);
          if (solved) {
            double tol = confirm ? std::min(opt.pcg_tolerance, iter_tol) : opt.pcg_tolerance;
            uint64_t limit = confirm ? opt.pcg_max_iterations : std::min<uint64_t>(opt.pcg_max_iterations, (uint64_t)D);
            // the explicit S is FP64 in both precisions, so its PCG needs no FP32 refinement loop
            PcgResult r = mixed && !explicit_op ? pcg_mixed(lambda, limit, tol) : pcg(lambda, limit, tol);
            pcg_terms += r.terms;
            solved = r.accepted;
            iterative_step = true;
            rel_res = r.rel;
            // Auto operator: once a PCG run needs many products, rebuilding the explicit S every
            // assembly costs less than the tile products it replaces. The switch waits for the next
            // assembly: this step's model reduction still needs the operator it was solved with.
            if (opt.matvec == 0 && !explicit_op && r.terms >= kExplicitSwitchTerms) switch_pending = true;
          }
        }
        double t2 = now();
        t_solve += t2 - t1;
        if (!solved) {
          rej[1]++;
          increase();
          continue;
        }
        // step cap (calibrated only)
        if (!n.self_cal && D > 0) {
          OMVGBA_LAUNCH(k_step_block_norm, grid_for(n.ncam, 128), 128, 0, st, n.ncam, d_pose_off.p, d_pose_dim.p, d_step.p,
                                                                   d_cam_norm.p);
          check_launch();
          std::vector<double> norms(n.ncam);
          CUDA_OK(copy_async(norms.data(), d_cam_norm.p, sizeof(double) * n.ncam, cudaMemcpyDeviceToHost, st));
          sync();
          double largest = 0.0;
          for (double x : norms) largest = std::max(largest, x);
          if (largest > 0.5) {
            OMVGBA_LAUNCH(k_scale, grid_for(D, 256), 256, 0, st, D, 0.5 / largest, d_step.p);
            check_launch();
          }
        }
        DevView v = view();
        OMVGBA_LAUNCH(k_retract, grid_for(std::max(n.ncam, ng), 128), 128, 0, st, v, ng, d_step.p, g, d_pose[cur].p,
                      d_groups[cur].p, d_pose[cand].p, d_groups[cand].p);
        if (mixed)
          OMVGBA_LAUNCH(k_candidate_points<float>, grid_for(P, 128), 128, 0, st, v, lin32(), d_step.p, state(cur),
                        state(cand), g, stages[si].loss, d_cand.p);
        else
          OMVGBA_LAUNCH(k_candidate_points<T>, grid_for(P, 128), 128, 0, st, v, lin(), d_step.p, state(cur),
                        state(cand), g, stages[si].loss, d_cand.p);
        check_launch();
        RedVec<4> cr = reduce<4>(d_cand.p, P, d_cand_part);
        if (cr.v[3] > 0.0) {
          rej[2]++;
          increase();
          t_candidate += now() - t2;
          continue;
        }
        double point_rms =
            std::sqrt(cr.v[1] / double(n.self_cal ? std::max(P, 1) : std::max<size_t>(free_points, 1)));
        // model reduction (camera_step.rs:44-81, optimizer.rs:590-618, retained/mod.rs:742-800)
        double damped;
        if (!iterative_step) {
          if (D > 0)
            rows_matvec(d_step.p, d_q.p, lambda);
          else
            CUDA_OK(cudaMemsetAsync(d_q.p, 0, sizeof(double), st));
        } else {
          matvec(d_step.p, d_q.p, lambda);
        }
        double h[4] = {0, 0, 0, 0};
        if (D > 0) dots({{d_gred.p, d_step.p}, {d_step.p, d_q.p}}, h);
        if (!iterative_step) {
          damped = a.point_red - h[0] - 0.5 * h[1];
        } else {
          damped = a.point_red + (-h[0] - 0.5 * h[1]);
          if (!(std::isfinite(damped) && damped > 0.0)) damped = NAN;
        }
        // camera damping norm: sum diag * step^2
        CUDA_OK(copy_async(d_tmp.p, d_step.p, sizeof(double) * std::max(D, 1), cudaMemcpyDeviceToDevice, st));
        double cd[1] = {0.0};
        if (D > 0) {
          std::vector<double> hs(D), hd(D);
          CUDA_OK(copy_async(hs.data(), d_step.p, sizeof(double) * D, cudaMemcpyDeviceToHost, st));
          CUDA_OK(copy_async(hd.data(), d_diag.p, sizeof(double) * D, cudaMemcpyDeviceToHost, st));
          sync();
          for (int i = 0; i < D; ++i) cd[0] += hd[i] * hs[i] * hs[i];
          double ss = 0.0;
          for (int i = 0; i < D; ++i) ss += hs[i] * hs[i];
          h[2] = ss;
        }
        double predicted = damped + 0.5 * lambda * (cd[0] + cr.v[2]);
        t_candidate += now() - t2;
        double reduction = current - cr.v[0];
        // NielsenController::accept
        double gain = (std::isfinite(reduction) && std::isfinite(predicted) && predicted > 0.0) ? reduction / predicted
                                                                                              : NAN;
        if (!(std::isfinite(gain) && gain > 0.0)) {
          increase();
          rej[3]++;
          continue;
        }
        double c2 = 2.0 * gain - 1.0;
        lambda = std::max(lambda * std::max(1.0 - c2 * c2 * c2, 1.0 / 3.0), 1e-12);
        nu = 2.0;
        std::swap(cur, cand);
        accepted++;
        double crms = std::sqrt(h[2] / double(std::max(D, 1)));
        double sn = std::sqrt(crms * crms + point_rms * point_rms);
        if (si == target) {
          target_accepted++;
          double relc = reduction / (1.0 + std::fabs(current));
          int cc = sn <= opt.step_tolerance ? 2 : (relc <= opt.relative_cost_tolerance ? 0 : -1);
          if (iterative_step && cc >= 0 && rel_res > iter_tol) {
            confirm = true;
            convergence = -1;
          } else {
            confirm = false;
            convergence = cc;
            if (cc >= 0) {
              done = true;
              break;
            }
          }
        }
      }
    }
    // final undamped assembly and certificate: the camera rank (sparse/direct.rs:288-455) and, for
    // self-calibration, the intrinsic marginal covariances (native/self_calibration.rs:255-303)
    const bool timing = std::getenv("OMVGBA_PHASE_TIMES") != nullptr;
    double tc = now();
    Gauge g = gauge_for(cur, scene);
    Assembly fa = assemble(cur, g, opt.loss, 0.0, true);
    if (timing) sync();
    const double t_final_assembly = now() - tc;
    tc = now();
    bool factored_s = false;
    if (!fa.valid)
      rep.rank = 2;
    else
      rep.rank = rank_certificate(&factored_s);
    const double t_rank = now() - tc;
    tc = now();
    if (n.self_cal && opt.certify_intrinsics) {
      rep.marginals_ok = fa.valid && intrinsic_marginals(factored_s, rep.marginals) ? 1 : 0;
    }
    if (timing)
      std::fprintf(stderr, "[omvgba] certificate: final assembly %.4fs rank %.4fs marginals %.4fs (nt %d bwt %d)\n",
                   t_final_assembly, t_rank, now() - tc, S.nt, S.bwt);
    bool well = rep.rank != 2 && fa.weak == 0;
    if (std::getenv("OMVGBA_PHASE_TIMES"))
      std::fprintf(stderr, "[omvgba] final: valid=%d rank=%d weak=%llu D=%d min_rcond=%.3e cost=%.12e\n", (int)fa.valid,
                   rep.rank, (unsigned long long)fa.weak, D, fa.min_rcond, fa.cost);
    if (!well)
      rep.status = 3;
    else if (convergence >= 0)
      rep.status = 0;
    else if (iterations > 0 && target_accepted == 0)
      rep.status = 2;
    else
      rep.status = 1;
    rep.reason = convergence;
    if (fa.valid) {
      rep.final_cost = fa.cost;
      rep.final_rmse = std::sqrt(fa.sq / double(2 * (size_t)N));
    } else {
      metrics(cur, opt.loss, &rep.final_cost, &rep.final_rmse);
    }
    rep.gradient_inf_norm = fa.grad_norm;
    rep.initial_cost = init_cost;
    rep.initial_rmse = init_rmse;
    rep.iterations = iterations;
    rep.accepted = accepted;
    for (int k = 0; k < 4; ++k) rep.rej[k] = rej[k];
    rep.rejected = rej[0] + rej[1] + rej[2] + rej[3];
    rep.weak = fa.weak;
    {
      OMVGBA_LAUNCH(k_noninvertible, grid_for(N, 256), 256, 0, st, view(), N, d_groups[cur].p, d_one.p);
      check_launch();
      RedVec<1> r = reduce<1>(d_one.p, N, d_one_part);
      rep.noninvertible = (uint64_t)r.v[0];
    }
    rep.pcg_terms = pcg_terms;
    rep.final_damping = lambda;
    rep.iterative = direct ? 0 : 1;
    if (std::getenv("OMVGBA_PHASE_TIMES"))
      std::fprintf(stderr,
                   "[omvgba] assemble %.3fs solve %.3fs candidate %.3fs total %.3fs pcg_terms %llu rejections "
                   "lin %llu solve %llu cand %llu gain %llu\n",
                   t_assemble, t_solve, t_candidate, now() - t_begin, (unsigned long long)pcg_terms,
                   (unsigned long long)rej[0], (unsigned long long)rej[1], (unsigned long long)rej[2],
                   (unsigned long long)rej[3]);
    rep.D = D;
    const double t_download = now();
    // download state
    std::vector<double> pose(12 * (size_t)n.ncam);
    CUDA_OK(copy_async(pose.data(), d_pose[cur].p, sizeof(double) * pose.size(), cudaMemcpyDeviceToHost, st));
    points.resize(n.points.size());
    CUDA_OK(copy_async(points.data(), d_points[cur].p, sizeof(double) * points.size(), cudaMemcpyDeviceToHost, st));
    groups.assign(n.groups.size(), 0.0);
    if (!groups.empty())
      CUDA_OK(copy_async(groups.data(), d_groups[cur].p, sizeof(double) * groups.size(), cudaMemcpyDeviceToHost, st));
    sync();
    rotation.resize(9 * (size_t)n.ncam);
    translation.resize(3 * (size_t)n.ncam);
    for (int c = 0; c < n.ncam; ++c) {
      for (int k = 0; k < 9; ++k) rotation[9 * c + k] = pose[12 * c + k];
      for (int k = 0; k < 3; ++k) translation[3 * c + k] = pose[12 * c + 9 + k];
    }
    if (std::getenv("OMVGBA_PHASE_TIMES")) std::fprintf(stderr, "[omvgba] download %.3fs\n", now() - t_download);
    return rep;
  }

};

// ---- two-view LM (kernel/two_view/optimizer.rs:16-240) -----------------------------------------
namespace {
// solve_positive_definite (numerics/refine/solver.rs:281-335) on the 5 x 5 reduced camera system
bool tv_solve_spd(const double A[25], const double b[5], double x[5]) {
  for (int i = 0; i < 25; ++i)
    if (!std::isfinite(A[i])) return false;
  for (int i = 0; i < 5; ++i)
    if (!std::isfinite(b[i])) return false;
  double L[5][5] = {};
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j <= i; ++j) {
      double acc = 0.0;
      for (int k = 0; k < j; ++k) acc += L[i][k] * L[j][k];
      const double sum = A[5 * i + j] - acc;
      if (!std::isfinite(sum)) return false;
      if (i == j) {
        if (sum <= 0.0) return false;
        L[i][j] = std::sqrt(sum);
      } else {
        L[i][j] = sum / L[j][j];
      }
    }
  double y[5];
  for (int i = 0; i < 5; ++i) {
    double sum = b[i];
    for (int j = 0; j < i; ++j) sum -= L[i][j] * y[j];
    y[i] = sum / L[i][i];
  }
  for (int i = 4; i >= 0; --i) {
    double sum = y[i];
    for (int j = i + 1; j < 5; ++j) sum -= L[j][i] * x[j];
    x[i] = sum / L[i][i];
  }
  for (int i = 0; i < 5; ++i)
    if (!std::isfinite(x[i])) return false;
  return true;
}
// the camera rank of the final system (schur.rs:338-370): eigenvalues of the symmetrized 5 x 5 by
// cyclic Jacobi rotations, counted above 64 eps n lambda_max
int tv_rank(const double H[25]) {
  double A[25];
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 5; ++j) A[5 * i + j] = 0.5 * (H[5 * i + j] + H[5 * j + i]);
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, scale = 0.0;
    for (int i = 0; i < 5; ++i) {
      scale = std::max(scale, std::fabs(A[6 * i]));
      for (int j = i + 1; j < 5; ++j) off += A[5 * i + j] * A[5 * i + j];
    }
    if (!(off > 1e-32 * scale * scale)) break;
    for (int p = 0; p < 5; ++p)
      for (int q = p + 1; q < 5; ++q) {
        const double apq = A[5 * p + q];
        if (apq == 0.0) continue;
        const double theta = (A[5 * q + q] - A[5 * p + p]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
        for (int k = 0; k < 5; ++k) {
          const double akp = A[5 * k + p], akq = A[5 * k + q];
          A[5 * k + p] = c * akp - sn * akq;
          A[5 * k + q] = sn * akp + c * akq;
        }
        for (int k = 0; k < 5; ++k) {
          const double apk = A[5 * p + k], aqk = A[5 * q + k];
          A[5 * p + k] = c * apk - sn * aqk;
          A[5 * q + k] = sn * apk + c * aqk;
        }
      }
  }
  double largest = 0.0;
  for (int i = 0; i < 5; ++i) largest = std::max(largest, std::fabs(A[6 * i]));
  if (!(std::isfinite(largest) && largest > 0.0)) return 0;
  const double tol = 64.0 * kEps * 5.0 * largest;
  int rank = 0;
  for (int i = 0; i < 5; ++i) rank += (std::isfinite(A[6 * i]) && A[6 * i] > tol) ? 1 : 0;
  return rank;
}
void tv_basis(const double t[3], double baseline, double dir[3], double b0[3], double b1[3]) {
  for (int k = 0; k < 3; ++k) dir[k] = t[k] / baseline;
  // s2_tangent_basis (numerics/manifold.rs:118-131)
  const double nv = std::sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
  const double u[3] = {dir[0] / nv, dir[1] / nv, dir[2] / nv};
  double ref[3] = {0, 0, 0};
  if (std::fabs(u[0]) <= std::fabs(u[1]) && std::fabs(u[0]) <= std::fabs(u[2]))
    ref[0] = 1;
  else if (std::fabs(u[1]) <= std::fabs(u[2]))
    ref[1] = 1;
  else
    ref[2] = 1;
  double a[3] = {u[1] * ref[2] - u[2] * ref[1], u[2] * ref[0] - u[0] * ref[2], u[0] * ref[1] - u[1] * ref[0]};
  const double na = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  for (int k = 0; k < 3; ++k) b0[k] = a[k] / na;
  b1[0] = u[1] * b0[2] - u[2] * b0[1];
  b1[1] = u[2] * b0[0] - u[0] * b0[2];
  b1[2] = u[0] * b0[1] - u[1] * b0[0];
}
}  // namespace

TwoViewReport gpu_two_view(Context* ctx, TwoViewProblem& pr, const LmOptions& opt) {
  CUDA_OK(cudaSetDevice(ctx->device));
  cudaStream_t st = opt.stream ? static_cast<cudaStream_t>(opt.stream) : ctx->stream;
  const int P = (int)(pr.points.size() / 3);
  if (P < 5) throw SolveFailure{OMVGBA_NUMERICAL, "two-view bundle adjustment needs at least 5 points"};
  double baseline = std::sqrt(pr.t[0] * pr.t[0] + pr.t[1] * pr.t[1] + pr.t[2] * pr.t[2]);
  if (!(std::isfinite(pr.t[0]) && std::isfinite(pr.t[1]) && std::isfinite(pr.t[2])) ||
      !(std::isfinite(baseline) && baseline > 64.0 * kEps))
    throw SolveFailure{OMVGBA_NUMERICAL, "two-view bundle adjustment translation is invalid"};
  DBuf<double> d_points, d_moved, d_obs, d_bearing, d_out, d_local, d_cand, d_sum, d_step;
  d_points.upload(pr.points.data(), pr.points.size(), st);
  d_moved.alloc(pr.points.size(), st);
  if (pr.angular)
    d_bearing.upload(pr.bearing.data(), pr.bearing.size(), st);
  else
    d_obs.upload(pr.obs.data(), pr.obs.size(), st);
  d_out.alloc((size_t)kTvOut * P, st);
  d_local.alloc((size_t)kTvLocal * P, st);
  d_cand.alloc((size_t)4 * P, st);
  d_sum.alloc(kTvOut, st);
  d_step.alloc(5, st);
  TvDev dev{};
  dev.P = P;
  dev.angular = pr.angular ? 1 : 0;
  std::memcpy(dev.cam, pr.cam, sizeof(dev.cam));
  dev.obs = d_obs.p;
  dev.bearing = d_bearing.p;
  TvPose pose{};
  std::memcpy(pose.R, pr.R, sizeof(pose.R));
  std::memcpy(pose.t, pr.t, sizeof(pose.t));
  const int grid = grid_for(P, 128);
  // one linearization + reduction: sums[0..42], max point gradient, min rcond, weak, invalid, failed
  auto system = [&](const TvPose& ps, const LossDev& loss, double lambda, double sums[kTvOut]) {
    double dir[3], b0[3], b1[3];
    tv_basis(ps.t, baseline, dir, b0, b1);
    OMVGBA_LAUNCH(k_tv_linearize, grid, 128, 0, st, dev, (const double*)d_points.p, ps, b0[0], b0[1], b0[2], b1[0],
                  b1[1], b1[2], baseline, loss, lambda, d_out.p, d_local.p);
    OMVGBA_LAUNCH(k_tv_reduce, 1, 1024, 0, st, (const double*)d_out.p, P, kTvOut, kTvSums, d_sum.p);
    CUDA_OK(cudaGetLastError());
    CUDA_OK(copy_async(sums, d_sum.p, sizeof(double) * kTvOut, cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    return sums[kTvSums + 4] == 0.0;  // every point projected in both views
  };
  auto floor_of = [](const double* diag) {
    double sc = 0.0;
    for (int k = 0; k < 5; ++k) sc = std::max(sc, diag[k]);
    return 64.0 * kEps * std::max(sc, kMinPositive);
  };
  auto scaled_ginf5 = [](const double* g, const double* diag) {
    double scale = 0.0;
    for (int i = 0; i < 5; ++i) scale = std::max(scale, diag[i]);
    if (!(std::isfinite(scale) && scale > 0.0)) {
      for (int i = 0; i < 5; ++i)
        if (g[i] != 0.0) return (double)INFINITY;
      return 0.0;
    }
    const double fl = 64.0 * kEps * scale;
    double best = 0.0;
    for (int i = 0; i < 5; ++i) best = std::max(best, std::fabs(g[i]) / std::sqrt(std::max(diag[i], fl)));
    return best;
  };
  auto valid_system = [](const double* s) {  // ReducedSystem::is_valid (schur.rs:151-155)
    if (s[kTvSums + 3] != 0.0) return false;
    for (int k = 0; k < 30; ++k)
      if (!std::isfinite(s[k])) return false;
    return true;
  };
  TwoViewReport rep;
  double sums[kTvOut];
  if (!system(pose, opt.loss, 0.0, sums))  // validate_projection_domain (optimizer.rs:396-415)
    throw SolveFailure{OMVGBA_NUMERICAL, "two-view bundle adjustment: a point is not projectable in both views"};
  rep.initial_cost = sums[40];
  rep.initial_rmse = std::sqrt(sums[41] / double(4 * (size_t)P));
  // stages (continuation.rs:18-74)
  struct StageLoss {
    LossDev loss;
    uint64_t iters;
  } stages[3];
  const LossDev l2{kLossL2, 0.0};
  if (opt.loss.kind == kLossCauchy) {
    const uint64_t w = std::min<uint64_t>(opt.max_iterations / 4, 5);
    stages[0] = {l2, w};
    stages[1] = {opt.loss, opt.max_iterations - w};
    stages[2] = {l2, 0};
  } else {
    stages[0] = {opt.loss, opt.max_iterations};
    stages[1] = {l2, 0};
    stages[2] = {l2, 0};
  }
  int target = 0;
  for (int i = 2; i >= 0; --i)
    if (stages[i].iters > 0) {
      target = i;
      break;
    }
  // LM run state (run_state.rs) with Nielsen damping (controller.rs:63-90), initial 1e-4
  double lambda = 1e-4, nu = 2.0;
  auto increase = [&]() {
    lambda = std::min(lambda * nu, 1e12);
    nu = std::min(nu * 2.0, 1e12);
  };
  uint64_t target_accepted = 0;
  int convergence = -1;
  bool done = false;
  for (int si = 0; si < 3 && !done; ++si) {
    for (uint64_t it = 0; it < stages[si].iters; ++it) {
      rep.iterations++;
      const double trial = lambda;
      if (!system(pose, stages[si].loss, trial, sums) || !valid_system(sums)) {
        rep.rej[0]++;
        increase();
        continue;
      }
      double H[25], g[5];
      std::memcpy(H, sums, sizeof(H));
      std::memcpy(g, sums + 25, sizeof(g));
      const double* full_g = sums + 30;
      const double* diag = sums + 35;
      const double fl = floor_of(diag);
      for (int k = 0; k < 5; ++k) H[6 * k] += trial * std::max(diag[k], fl);  // finish_damping
      const double current = sums[40];
      const double gnorm = std::max(sums[kTvSums], scaled_ginf5(full_g, diag));
      if (si == target && convergence < 0 && std::isfinite(gnorm) && gnorm >= 0.0 && std::isfinite(current) &&
          gnorm <= opt.gradient_tolerance * (1.0 + std::fabs(current))) {
        convergence = 1;
        done = true;
        break;
      }
      double raw[5], step[5];
      if (!tv_solve_spd(H, g, raw)) {
        rep.rej[1]++;
        increase();
        continue;
      }
      for (int k = 0; k < 5; ++k) step[k] = -raw[k];
      {  // limit_pose_step (optimizer.rs:432-443)
        const double rn = std::sqrt(step[0] * step[0] + step[1] * step[1] + step[2] * step[2]);
        const double tn = std::sqrt(step[3] * step[3] + step[4] * step[4]);
        const double len = std::max(rn, tn);
        if (len > 0.5)
          for (double& v : step) v *= 0.5 / len;
      }
      // retract_pose (optimizer.rs:365-381)
      double dir[3], b0[3], b1[3];
      tv_basis(pose.t, baseline, dir, b0, b1);
      TvPose cand{};
      {
        double w[3] = {step[0], step[1], step[2]}, U[9];
        exp_so3_dev(w, U);
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            double acc = 0.0;
            for (int k = 0; k < 3; ++k) acc += U[3 * i + k] * pose.R[3 * k + j];
            cand.R[3 * i + j] = acc;
          }
        // retract_s2 (numerics/manifold.rs:133-147)
        const double vv[3] = {b0[0] * step[3] + b1[0] * step[4], b0[1] * step[3] + b1[1] * step[4],
                              b0[2] * step[3] + b1[2] * step[4]};
        const double th = std::sqrt(vv[0] * vv[0] + vv[1] * vv[1] + vv[2] * vv[2]);
        const double tn = std::sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
        const double tv[3] = {dir[0] / tn, dir[1] / tn, dir[2] / tn};
        double nd[3];
        if (th < 1e-10) {
          const double sv[3] = {tv[0] + vv[0], tv[1] + vv[1], tv[2] + vv[2]};
          const double nn = std::sqrt(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]);
          for (int k = 0; k < 3; ++k) nd[k] = sv[k] / nn;
        } else {
          const double cs = std::cos(th), sn = std::sin(th) / th;
          for (int k = 0; k < 3; ++k) nd[k] = tv[k] * cs + vv[k] * sn;
        }
        for (int k = 0; k < 3; ++k) cand.t[k] = baseline * nd[k];
      }
      CUDA_OK(copy_async(d_step.p, step, sizeof(step), cudaMemcpyHostToDevice, st));
      OMVGBA_LAUNCH(k_tv_candidate, grid, 128, 0, st, dev, (const double*)d_points.p, (const double*)d_local.p, trial,
                    (const double*)d_step.p, cand, baseline, stages[si].loss, d_moved.p, d_cand.p);
      OMVGBA_LAUNCH(k_tv_reduce, 1, 1024, 0, st, (const double*)d_cand.p, P, 4, 4, d_sum.p);
      CUDA_OK(cudaGetLastError());
      double cs[4];
      CUDA_OK(copy_async(cs, d_sum.p, sizeof(cs), cudaMemcpyDeviceToHost, st));
      CUDA_OK(cudaStreamSynchronize(st));
      if (cs[3] != 0.0) {
        rep.rej[2]++;
        increase();
        continue;
      }
      const double point_rms = std::sqrt(cs[1] / double(P));
      const double reduction = current - cs[0];
      // ReducedSystem::predicted_reduction (schur.rs:161-196), with the damped camera system
      double quad = 0.0, gs = 0.0, pdn = 0.0;
      for (int r = 0; r < 5; ++r) {
        double hs = 0.0;
        for (int c = 0; c < 5; ++c) hs += H[5 * r + c] * step[c];
        quad += step[r] * hs;
      }
      for (int r = 0; r < 5; ++r) gs += g[r] * step[r];
      for (int r = 0; r < 5; ++r) pdn += std::max(diag[r], fl) * step[r] * step[r];
      const double predicted = (sums[42] - gs - 0.5 * quad) + 0.5 * trial * (pdn + cs[2]);
      // NielsenController::accept (controller.rs:63-90)
      const double gain = (std::isfinite(reduction) && std::isfinite(predicted) && predicted > 0.0)
                              ? reduction / predicted
                              : std::nan("");
      if (!(std::isfinite(gain) && gain > 0.0)) {
        rep.rej[3]++;
        increase();
        continue;
      }
      const double c3 = 2.0 * gain - 1.0;
      lambda = std::max(lambda * std::max(1.0 - c3 * c3 * c3, 1.0 / 3.0), 1e-12);
      nu = 2.0;
      // commit_points: the moved points of this step (the same back-substitution at the same state)
      CUDA_OK(cudaMemcpyAsync(d_points.p, d_moved.p, sizeof(double) * 3 * (size_t)P, cudaMemcpyDeviceToDevice, st));
      pose = cand;
      rep.accepted++;
      double ss = 0.0;
      for (double v : step) ss += v * v;
      const double prms = std::sqrt(ss / 5.0);
      const double sn = std::sqrt(prms * prms + point_rms * point_rms);
      if (si == target) {
        target_accepted++;
        const double rel = reduction / (1.0 + std::fabs(current));
        const int cc = sn <= opt.step_tolerance ? 2 : (rel <= opt.relative_cost_tolerance ? 0 : -1);
        convergence = cc;
        if (cc >= 0) {
          done = true;
          break;
        }
      }
    }
  }
  // the final undamped system
  const bool have = system(pose, opt.loss, 0.0, sums);
  double Hf[25];
  std::memcpy(Hf, sums, sizeof(Hf));
  const bool valid = have && valid_system(sums);
  rep.rank = valid ? tv_rank(Hf) : 0;
  rep.weak = have ? (uint64_t)sums[kTvSums + 2] : (uint64_t)P;
  const bool well = rep.rank == 5 && rep.weak == 0;
  rep.status = !well ? 3 : (convergence >= 0 ? 0 : (rep.iterations > 0 && target_accepted == 0 ? 2 : 1));
  rep.reason = convergence;
  rep.grad_norm = valid ? std::max(sums[kTvSums], scaled_ginf5(sums + 30, sums + 35)) : INFINITY;
  if (have) {
    rep.final_cost = sums[40];
    rep.final_rmse = std::sqrt(sums[41] / double(4 * (size_t)P));
  } else {  // metrics (schur.rs:303-330): a point that no longer projects makes both infinite
    rep.final_cost = INFINITY;
    rep.final_rmse = INFINITY;
  }
  rep.final_damping = lambda;
  std::memcpy(rep.R, pose.R, sizeof(rep.R));
  std::memcpy(rep.t, pose.t, sizeof(rep.t));
  CUDA_OK(copy_async(pr.points.data(), d_points.p, sizeof(double) * 3 * (size_t)P, cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaStreamSynchronize(st));
  return rep;
}

NativeReport gpu_refine(Context* ctx, const NativeProblem& problem, const LmOptions& options,
                        std::vector<double>& rotation, std::vector<double>& translation, std::vector<double>& points,
                        std::vector<double>& groups) {
  CUDA_OK(cudaSetDevice(ctx->device));
  if (problem.obs_cam.size() >= (1ull << 31)) throw SolveFailure{3, "observation count exceeds 2^31"};
  Solver<double> s(ctx, problem, options);
  return s.refine(rotation, translation, points, groups);
}

struct Resident {
  Context* ctx = nullptr;
  Solver<double>* solver = nullptr;
  bool linearized = false;  // the records hold the initial state's linearization at `lambda`
  double lambda = 0.0;
  ~Resident() { delete solver; }
};

Resident* resident_create(Context* ctx, const NativeProblem& problem, const LmOptions& options) {
  CUDA_OK(cudaSetDevice(ctx->device));
  if (problem.obs_cam.size() >= (1ull << 31)) throw SolveFailure{3, "observation count exceeds 2^31"};
  Resident* r = new Resident();
  r->ctx = ctx;
  try {
    r->solver = new Solver<double>(ctx, problem, options);
    r->solver->keep_initial();
    r->solver->sync();
  } catch (...) {
    delete r;
    throw;
  }
  return r;
}

void resident_destroy(Resident* r) {
  if (!r) return;
  cudaSetDevice(r->ctx->device);
  cudaStream_t st = r->solver ? r->solver->st : nullptr;
  delete r;
  if (st) cudaStreamSynchronize(st);
}

NativeReport resident_refine(Resident* r, std::vector<double>& rotation, std::vector<double>& translation,
                             std::vector<double>& points, std::vector<double>& groups) {
  CUDA_OK(cudaSetDevice(r->ctx->device));
  r->linearized = false;
  r->solver->restore_initial();
  return r->solver->refine(rotation, translation, points, groups);
}

ResidentInfo resident_info(const Resident* r) {
  const Solver<double>& s = *r->solver;
  ResidentInfo info;
  info.observations = (uint64_t)s.N;
  info.points = (uint64_t)s.P;
  info.cameras = (uint64_t)s.n.ncam;
  info.dimension = (uint64_t)s.D;
  info.iterative = s.direct ? 0 : 1;
  info.mixed = s.mixed ? 1 : 0;
  for (int p = 0; p < s.P; ++p) {
    const int point_dim = s.n.fixed_points[p] ? 0 : 3;
    for (uint64_t o = s.n.pt_off[p]; o < s.n.pt_off[p + 1]; ++o) {
      const int c = (int)s.n.obs_cam[o];
      int cam_dim = s.L.pose_dim[c];
      if (s.n.self_cal) cam_dim += s.L.intr_dim[s.n.cam_group[c]];
      info.jacobian_entries += 2 * (uint64_t)(cam_dim + point_dim);
    }
  }
  info.tiles64 = s.mixed ? 0 : (uint64_t)s.dT64.ntiles;
  info.tiles32 = s.mixed ? (uint64_t)s.dT32.ntiles : 0;
  info.record_bytes64 = sizeof(double) * s.d_rec.n;
  info.record_bytes32 = sizeof(float) * s.d_rec32.n;
  info.metadata_bytes64 = s.mixed ? 0 : s.dT64.slots.n + sizeof(uint32_t) * s.dT64.tile_hdr.n;
  info.metadata_bytes32 = s.mixed ? s.dT32.slots.n + sizeof(uint32_t) * s.dT32.tile_hdr.n : 0;
  return info;
}

void resident_schur_product(Resident* r, double lambda, bool fp32, int stage, const double* x, double* y) {
  CUDA_OK(cudaSetDevice(r->ctx->device));
  Solver<double>& s = *r->solver;
  if (s.direct) throw SolveFailure{2, "the plan's linear solver is direct; the tile product serves PCG plans"};
  if (fp32 && !s.mixed) throw SolveFailure{1, "FP32 products need a mixed-precision plan"};
  if (!r->linearized || r->lambda != lambda) {
    s.restore_initial();
    double scene = s.scene_scale_host();
    Gauge g = s.gauge_for(s.cur, scene);
    auto a = s.assemble(s.cur, g, s.opt.loss, lambda, false);
    if (!a.valid) throw SolveFailure{4, "linearization is not valid"};
    r->linearized = true;
    r->lambda = lambda;
  }
  if (stage == 1)
    s.matvec_tiles(x, nullptr, fp32);
  else if (stage == 2)
    s.build_rows();
  else if (stage == 3)
    s.camera_sums();
  else
    s.matvec(x, y, lambda, nullptr, fp32);
  s.check_launch();
}

void gpu_debug_linearize(Context* ctx, const NativeProblem& problem, const LmOptions& options, double* residual,
                         double* sqrt_weight, double* point_jacobian, double* camera_jacobian) {
  CUDA_OK(cudaSetDevice(ctx->device));
  Solver<double> s(ctx, problem, options);
  double scene = s.scene_scale_host();
  Gauge g = s.gauge_for(s.cur, scene);
  size_t N = problem.obs_cam.size();
  DBuf<double> d_sw;
  d_sw.alloc(std::max<size_t>(N, 1), s.st);
  LinOut<double> lo = s.lin();
  lo.sw = d_sw.p;
  const MvTiles mt = s.dT64.view(s.d_blk_dim.p, s.d_blk_off.p, s.nb);
  if (mt.ntiles > 0)
    OMVGBA_LAUNCH(k_linearize_tiles<double>, mt.ntiles, mv_tile_obs<double>(), 0, s.st, s.view(), s.state(s.cur), g,
                  options.loss, 0.0, lo, mt);
  s.check_launch();
  std::vector<double> rec(s.d_rec.n), rw(2 * N), sw(N);
  CUDA_OK(copy_async(rec.data(), s.d_rec.p, sizeof(double) * rec.size(), cudaMemcpyDeviceToHost, s.st));
  CUDA_OK(copy_async(rw.data(), s.d_rw.p, sizeof(double) * rw.size(), cudaMemcpyDeviceToHost, s.st));
  CUDA_OK(copy_async(sw.data(), d_sw.p, sizeof(double) * N, cudaMemcpyDeviceToHost, s.st));
  s.sync();
  // the kernel stores sqrt-weighted rows; divide the weight back out
  for (size_t o = 0; o < N; ++o) {
    double w = sw[o];
    sqrt_weight[o] = w;
    for (int k = 0; k < 2; ++k) residual[2 * o + k] = rw[2 * o + k] / w;
    const size_t base = s.T64.obs_rec[o], rs = (size_t)mv_tile_obs<double>();
    for (int k = 0; k < 6; ++k) point_jacobian[6 * o + k] = rec[base + (kJp + k) * rs] / w;
    for (int k = 0; k < 18; ++k) camera_jacobian[18 * o + k] = rec[base + k * rs] / w;
  }
}

// Debug: y_mv = S_lambda x by the matrix-free tile kernel and y_dense = S_lambda x from the explicit
// dense Schur complement, both at the first linearization (FP64), for operator parity tests.
void gpu_debug_schur_product(Context* ctx, const NativeProblem& problem, const LmOptions& options, double lambda,
                             const double* x, double* y_mv, double* y_dense, int* dimension) {
  CUDA_OK(cudaSetDevice(ctx->device));
  LmOptions o = options;
  o.iterative = false;
  o.linear_solver = 1;
  Solver<double> s(ctx, problem, o);
  double scene = s.scene_scale_host();
  Gauge g = s.gauge_for(s.cur, scene);
  auto a = s.assemble(s.cur, g, options.loss, lambda, true);
  if (!a.valid) throw SolveFailure{4, "linearization is not valid"};
  int D = s.D;
  *dimension = D;
  if (!x) return;
  CUDA_OK(copy_async(s.d_tmp.p, x, sizeof(double) * D, cudaMemcpyHostToDevice, s.st));
  s.matvec(s.d_tmp.p, s.d_q.p, lambda);
  s.rows_matvec(s.d_tmp.p, s.d_z.p, lambda);
  CUDA_OK(copy_async(y_mv, s.d_q.p, sizeof(double) * D, cudaMemcpyDeviceToHost, s.st));
  CUDA_OK(copy_async(y_dense, s.d_z.p, sizeof(double) * D, cudaMemcpyDeviceToHost, s.st));
  s.sync();
}

}  // namespace omvgba
