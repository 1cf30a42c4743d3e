// mv_tiles.cuh — matrix-free reduced-camera-system product y = S_lambda x for the PCG loop.
//
// S x = sum_o Jc_o^T (e_o - Jp_o z_p) + lambda diag x, with e_o = Jc_o x and
// z_p = Vhat_p^-1 sum_o Jp_o^T e_o (retained/operator.rs:137-227 computes the same product from
// cached Vhat^-1 W^T rows).
//
// Layout: observations are point-major; a tile is a run of whole points with at most TILE
// observations. Everything a tile needs is contiguous in HBM and 16 B aligned: its Jacobian
// records (component-major, so a warp's shared-memory reads are conflict-free), its points'
// damped inverses and a metadata blob built once per solve. A persistent CTA walks tiles with
// two shared-memory stages filled by bulk asynchronous copies (cp.async.bulk, one mbarrier per
// stage): every Jacobian byte crosses HBM once per product, and the next tile streams in while
// the current one is computed.
//
// Per tile, with a (tile, camera) "segment" for each camera the tile's observations see:
//   P0  x of each segment's pose and intrinsic parameters into shared memory (one gather per
//       segment and parameter instead of one per observation);
//   P1  thread per observation: e = Jc x, point terms Jp^T e;
//   P2  four lanes per point (one per component of the track sum, in track order, exchanged by
//       shuffles): z = Vhat^-1 (sum of the point terms);
//   P3  thread per observation: f = e - Jp z and its camera terms Jc^T f, stored in segment order;
//   P4  thread per (segment, parameter): the sum of the segment's contiguous run of camera terms,
//       in observation order, written as the segment's partial.
// The finalize kernel sums each block's partials in tile order (one warp per block, fixed lane
// assignment and shuffle tree) and adds lambda diag x. No sum depends on scheduling, so the
// product is bitwise reproducible run to run.
#pragma once

#include <cstdint>

namespace omvgba {

struct MvTiles {
  int ntiles;
  const uint32_t* tile_obs;     // ntiles + 1: first observation of each tile
  const uint32_t* tile_pt;      // ntiles + 1: first point of each tile
  const uint64_t* tile_blob;    // ntiles + 1: byte offset of each tile's metadata blob
  const unsigned char* blob;    // metadata blobs
  int nblocks;
  const int* blk_dim;
  const int* blk_off;
  const uint32_t* blk_seg_off;  // nblocks + 1
  const uint32_t* blk_segs;     // per block: (segment << 2) | column code, in tile order
};

// Metadata blob of a tile (header, then 16 B aligned sections):
//   u32 header[4] = {nobs, npt, nseg, seg_base}
//   u16 oseg[nobs]    segment of each observation
//   u16 lpt[nobs]     local point of each observation
//   u16 pos[nobs]     position of each observation in segment order
//   u16 poff[npt+1]   local observation range of each point
//   u16 segb[nseg+1]  range of each segment in ent
//   u32 w0[nseg]      pose parameter offset | pose dim << 28
//   u32 w1[nseg]      intrinsic parameter offset | intrinsic dim << 28
struct BlobView {
  uint32_t nobs, npt, nseg, seg_base;
  const uint16_t* oseg;
  const uint16_t* lpt;
  const uint16_t* pos;
  const uint16_t* poff;
  const uint16_t* segb;
  const uint32_t* w0;
  const uint32_t* w1;
};
__host__ __device__ __forceinline__ size_t align16(size_t x) { return (x + 15) & ~size_t(15); }
// Section offsets of a blob with the given counts; returns the total (16 B multiple) size.
__host__ __device__ __forceinline__ size_t blob_layout(uint32_t nobs, uint32_t npt, uint32_t nseg, size_t off[7]) {
  size_t o = 16;
  off[0] = o;
  o = align16(o + 2 * (size_t)nobs);
  off[1] = o;
  o = align16(o + 2 * (size_t)nobs);
  off[2] = o;
  o = align16(o + 2 * (size_t)nobs);
  off[3] = o;
  o = align16(o + 2 * (size_t)(npt + 1));
  off[4] = o;
  o = align16(o + 2 * (size_t)(nseg + 1));
  off[5] = o;
  o = align16(o + 4 * (size_t)nseg);
  off[6] = o;
  o = align16(o + 4 * (size_t)nseg);
  return o;
}
__device__ __forceinline__ BlobView blob_view(const unsigned char* b) {
  BlobView v;
  const uint32_t* h = reinterpret_cast<const uint32_t*>(b);
  v.nobs = h[0];
  v.npt = h[1];
  v.nseg = h[2];
  v.seg_base = h[3];
  size_t off[7];
  blob_layout(v.nobs, v.npt, v.nseg, off);
  v.oseg = reinterpret_cast<const uint16_t*>(b + off[0]);
  v.lpt = reinterpret_cast<const uint16_t*>(b + off[1]);
  v.pos = reinterpret_cast<const uint16_t*>(b + off[2]);
  v.poff = reinterpret_cast<const uint16_t*>(b + off[3]);
  v.segb = reinterpret_cast<const uint16_t*>(b + off[4]);
  v.w0 = reinterpret_cast<const uint32_t*>(b + off[5]);
  v.w1 = reinterpret_cast<const uint32_t*>(b + off[6]);
  return v;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// Arrival that arms the barrier for `bytes` of transactions (a plain arrival when zero).
__device__ __forceinline__ void mbar_arrive_expect(uint64_t* bar, uint32_t bytes) {
  if (bytes == 0)
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
  else
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// One bulk copy global -> own shared memory (no multicast), completing on `bar`. bytes % 16 == 0.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  if (bytes == 0) return;
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
// Bounded wait for phase `parity` of the barrier; false after the iteration limit.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  uint32_t a = smem_addr(bar);
  for (int it = 0; it < (1 << 24); ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

constexpr int kMvThreads = 256;
constexpr int kSegParams = 9;  // pose (<= 6) then intrinsic (<= 3) parameters of a segment

template <typename T>
__host__ __device__ constexpr int mv_tile_obs() {
  return sizeof(T) == 4 ? 256 : 128;
}
// Upper bound of a tile's metadata blob (npt <= nobs <= TILE, nseg <= TILE).
__host__ __device__ constexpr size_t mv_blob_max(int tile) { return 18 * (size_t)tile + 144; }
template <typename T>
__host__ __device__ constexpr size_t mv_stage_bytes() {
  return align16(sizeof(T) * (size_t)mv_tile_obs<T>() * kRec) + align16(mv_blob_max(mv_tile_obs<T>())) +
         48 * (size_t)mv_tile_obs<T>();
}
// Row stride of the per-observation term arrays: one element of padding, so the 9 lanes that
// read the 9 parameter rows of one observation hit 9 different banks.
template <typename T>
__host__ __device__ constexpr int mv_term_stride() {
  return mv_tile_obs<T>() + 1;
}
// Two stages, then x per segment (9 TILE), the point / camera terms (9 padded rows) and z (3 TILE).
template <typename T>
__host__ __device__ constexpr size_t mv_smem_bytes() {
  return 2 * mv_stage_bytes<T>() +
         sizeof(T) * ((size_t)mv_tile_obs<T>() * 12 + (size_t)kSegParams * mv_term_stride<T>() + 4);
}

__host__ __device__ __forceinline__ int colcode_to_col(int code) { return code == 0 ? 0 : (code == 1 ? 5 : 6); }

template <typename T>
__device__ __forceinline__ void mv_issue_tile(const MvTiles& mt, int t, const T* rec, const double* vinv,
                                              unsigned char* stage, uint64_t* bar) {
  constexpr int TILE = mv_tile_obs<T>();
  const uint32_t o0 = mt.tile_obs[t], o1 = mt.tile_obs[t + 1];
  const uint32_t p0 = mt.tile_pt[t], p1 = mt.tile_pt[t + 1];
  const uint64_t b0 = mt.tile_blob[t], b1 = mt.tile_blob[t + 1];
  const uint32_t rb = (o1 > o0 ? (uint32_t)TILE : 0u) * kRec * (uint32_t)sizeof(T);  // whole tile block
  const uint32_t bb = (uint32_t)(b1 - b0);
  const uint32_t vb = (p1 - p0) * 48u;
  mbar_arrive_expect(bar, rb + bb + vb);
  unsigned char* s_rec = stage;
  unsigned char* s_blob = stage + align16(sizeof(T) * (size_t)TILE * kRec);
  unsigned char* s_vinv = s_blob + align16(mv_blob_max(TILE));
  bulk_copy_g2s(s_rec, rec + (size_t)t * TILE * kRec, rb, bar);
  bulk_copy_g2s(s_blob, mt.blob + b0, bb, bar);
  bulk_copy_g2s(s_vinv, vinv + 6 * (size_t)p0, vb, bar);
}

template <typename T>
__global__ void __launch_bounds__(kMvThreads, 2)
    k_mv_tiles(MvTiles mt, const T* __restrict__ rec, const double* __restrict__ vinv, const double* __restrict__ x,
               double* __restrict__ partial, const PcgCtl* ctl, int* fault) {
  if (pcg_stopped(ctl)) return;
  constexpr int TILE = mv_tile_obs<T>();
  extern __shared__ __align__(128) unsigned char smem_raw[];
  constexpr int TS = mv_term_stride<T>();
  T* xs = reinterpret_cast<T*>(smem_raw + 2 * mv_stage_bytes<T>());  // kSegParams per segment
  T* zz = xs + kSegParams * TILE;                                    // z, component-major
  T* terms = zz + 3 * TILE;                                          // point terms, then camera terms
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ int abort_flag;
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
    abort_flag = 0;
  }
  __syncthreads();
  int t = blockIdx.x;
  if (t < mt.ntiles && tid == 0) {
    mv_issue_tile<T>(mt, t, rec, vinv, smem_raw, &bar[0]);
  }
  for (int k = 0; t < mt.ntiles; t += gridDim.x, ++k) {
    const int stage = k & 1;
    const int tn = t + gridDim.x;
    bool issued_next = false;
    if (tid == 0 && tn < mt.ntiles) {
      // the other stage was last read by the previous tile; order those reads before the async writes
      fence_proxy_async();
      mv_issue_tile<T>(mt, tn, rec, vinv, smem_raw + (stage ^ 1) * mv_stage_bytes<T>(), &bar[stage ^ 1]);
      issued_next = true;
    }
    // every thread observes the phase completion (acquire of the async-proxy writes), bounded
    if (!mbar_wait(&bar[stage], (uint32_t)((k >> 1) & 1))) abort_flag = 1;
    __syncthreads();
    if (abort_flag) {
      if (tid == 0) {
        atomicExch(fault, 1);
        if (issued_next) mbar_wait(&bar[stage ^ 1], (uint32_t)(((k + 1) >> 1) & 1));  // drain, bounded
      }
      return;
    }
    const unsigned char* sp = smem_raw + stage * mv_stage_bytes<T>();
    const T* cur = reinterpret_cast<const T*>(sp);
    const BlobView bv = blob_view(sp + align16(sizeof(T) * (size_t)TILE * kRec));
    const double* vi_s =
        reinterpret_cast<const double*>(sp + align16(sizeof(T) * (size_t)TILE * kRec) + align16(mv_blob_max(TILE)));
    const uint32_t nobs = bv.nobs, npt = bv.npt, nseg = bv.nseg;
    // P0: x of each segment's parameters (zero beyond the segment's dimensions)
    for (uint32_t w = tid; w < kSegParams * nseg; w += blockDim.x) {
      const uint32_t s = w / kSegParams, c = w - kSegParams * s;
      const uint32_t w0 = bv.w0[s], w1 = bv.w1[s];
      const uint32_t pd = w0 >> 28, id = w1 >> 28;
      double v = 0.0;
      if (c < pd)
        v = __ldg(x + (w0 & 0x0FFFFFFFu) + c);
      else if (c - pd < id)
        v = __ldg(x + (w1 & 0x0FFFFFFFu) + (c - pd));
      xs[w] = (T)v;
    }
    __syncthreads();
    // P1: e = Jc x and the point terms Jp^T e (record component k of observation i at k TILE + i)
    // The observation's Jacobian stays in registers until P3.
    T e0 = 0, e1 = 0, jc[18], jp[6];
    if ((uint32_t)tid < nobs) {
      const T* r = cur + tid;
      const T* xv = xs + kSegParams * bv.oseg[tid];
#pragma unroll
      for (int c = 0; c < 18; ++c) jc[c] = r[c * TILE];
#pragma unroll
      for (int c = 0; c < 6; ++c) jp[c] = r[(kJp + c) * TILE];
#pragma unroll
      for (int c = 0; c < 9; c += 2) {  // two accumulators per row: shorter dependency chains
        const T xa = xv[c];
        e0 += jc[c] * xa;
        e1 += jc[9 + c] * xa;
      }
      T e0b = 0, e1b = 0;
#pragma unroll
      for (int c = 1; c < 9; c += 2) {
        const T xb = xv[c];
        e0b += jc[c] * xb;
        e1b += jc[9 + c] * xb;
      }
      e0 += e0b;
      e1 += e1b;
      terms[tid] = jp[0] * e0 + jp[3] * e1;
      terms[TS + tid] = jp[1] * e0 + jp[4] * e1;
      terms[2 * TS + tid] = jp[2] * e0 + jp[5] * e1;
    }
    __syncthreads();
    // P2: z_p = Vhat_p^-1 sum_o Jp_o^T e_o; lanes 4q..4q+2 of a warp sum the three components of
    // point q's track (in track order), lane 4q+3 idles; the sums are exchanged by shuffles.
    for (uint32_t base = 0; base < npt; base += blockDim.x >> 2) {
      const uint32_t lp = base + (tid >> 2), k = tid & 3;
      const bool active = lp < npt && k < 3;
      T bk = 0;
      if (active) {
        const T* row = terms + k * TS;
        for (uint32_t i = bv.poff[lp]; i < bv.poff[lp + 1]; ++i) bk += row[i];
      }
      const int lead = (tid & 31) & ~3;
      const T b0 = __shfl_sync(0xffffffffu, bk, lead), b1 = __shfl_sync(0xffffffffu, bk, lead + 1),
              b2 = __shfl_sync(0xffffffffu, bk, lead + 2);
      if (active) {
        // row k of the packed symmetric inverse (0,0) (1,0) (1,1) (2,0) (2,1) (2,2)
        const double* vi = vi_s + 6 * (size_t)lp;
        const int i0 = k == 0 ? 0 : (k == 1 ? 1 : 3), i1 = k == 0 ? 1 : (k == 1 ? 2 : 4), i2 = k == 0 ? 3 : (k == 1 ? 4 : 5);
        zz[k * TILE + lp] = (T)vi[i0] * b0 + (T)vi[i1] * b1 + (T)vi[i2] * b2;
      }
    }
    __syncthreads();
    // P3: f = e - Jp z and the camera terms Jc^T f (overwrite the point terms, read in P2 only)
    if ((uint32_t)tid < nobs) {
      const uint32_t lp = bv.lpt[tid];
      const T z0 = zz[lp], z1 = zz[TILE + lp], z2 = zz[2 * TILE + lp];
      const T f0 = e0 - (jp[0] * z0 + jp[1] * z1 + jp[2] * z2);
      const T f1 = e1 - (jp[3] * z0 + jp[4] * z1 + jp[5] * z2);
      const uint32_t q = bv.pos[tid];
#pragma unroll
      for (int c = 0; c < 9; ++c) terms[c * TS + q] = jc[c] * f0 + jc[9 + c] * f1;
    }
    __syncthreads();
    // P4: per (segment, parameter) sum of the segment's run of camera terms in observation order
    for (uint32_t w = tid; w < kSegParams * nseg; w += blockDim.x) {
      const uint32_t s = w / kSegParams, c = w - kSegParams * s;
      if (c >= (bv.w0[s] >> 28) + (bv.w1[s] >> 28)) continue;
      T acc = 0;
      const T* col = terms + c * TS;
      for (uint32_t j = bv.segb[s]; j < bv.segb[s + 1]; ++j) acc += col[j];
      partial[(size_t)kSegParams * (bv.seg_base + s) + c] = (double)acc;
    }
    __syncthreads();
  }
}

// y_b = sum of block b's segment partials (tile order) + lambda diag_b x_b: one warp per block,
// lane l sums entries l, l + 32, ... in order, then a fixed shuffle tree.
__global__ void k_mv_tiles_finalize(MvTiles mt, const double* __restrict__ partial, const double* __restrict__ diag,
                                    double lambda, const double* __restrict__ x, double* __restrict__ y,
                                    const PcgCtl* ctl) {
  if (pcg_stopped(ctl)) return;
  const int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (b >= mt.nblocks) return;
  const int o = mt.blk_off[b], d = mt.blk_dim[b];
  const uint32_t i0 = mt.blk_seg_off[b], i1 = mt.blk_seg_off[b + 1];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (uint32_t i = i0 + lane; i < i1; i += 32) {
    const uint32_t e = mt.blk_segs[i];
    const double* pp = partial + (size_t)kSegParams * (e >> 2) + colcode_to_col((int)(e & 3u));
#pragma unroll
    for (int c = 0; c < 6; ++c)
      if (c < d) acc[c] += pp[c];
  }
#pragma unroll
  for (int c = 0; c < 6; ++c) acc[c] = warp_sum(acc[c]);  // full sums land in lane 0
  if (lane == 0) {
#pragma unroll
    for (int c = 0; c < 6; ++c)
      if (c < d) y[o + c] = acc[c] + lambda * diag[o + c] * x[o + c];
  }
}

}  // namespace omvgba
