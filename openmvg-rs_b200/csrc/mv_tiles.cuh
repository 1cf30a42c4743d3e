// mv_tiles.cuh — fused matrix-free reduced-camera-system product S x for the PCG hot loop.
//
// S x = sum_o Jc_o^T (e_o - Jp_o z_p)   with e_o = Jc_o x_o and z_p = Vhat_p^-1 sum_o Jp_o^T e_o,
// plus lambda * diag * x in the finalize (retained/operator.rs:137-227 computes the same product
// from cached Vhat^-1 W^T rows).
//
// Layout: observations are point-major; a tile is a run of whole points with at most TILE
// observations. Everything a tile needs is contiguous in HBM and 16 B aligned: its Jacobian
// records, its points' damped inverses, and a metadata blob (per-observation column offsets,
// local point indices, point ranges, block segments and their entities) built once per solve.
// A persistent CTA walks tiles with two shared-memory stages: while it computes one tile, the
// bulk async copies (cp.async.bulk, completion on one mbarrier per stage) stream the next, so
// every Jacobian byte crosses HBM once per product and no thread waits on a dependent load.
// Inside a tile: observation-parallel e_o, point-parallel z_p, observation-parallel f_o, and one
// thread per (tile, parameter block) segment summing its entities in a fixed order into a partial.
// The finalize sums each block's partials in tile order: the product is bitwise deterministic.
#pragma once

#include <cstdint>

namespace omvgba {

struct MvTiles {
  int ntiles;
  const uint32_t* tile_obs;    // ntiles + 1: first observation (record) of each tile
  const uint32_t* tile_pt;     // ntiles + 1: first point of each tile
  const uint64_t* tile_blob;   // ntiles + 1: byte offset of each tile's metadata blob
  const unsigned char* blob;   // metadata blobs
  const int* blk_dim;
  const int* blk_off;
  const uint32_t* blk_seg_off;  // nblocks + 1
  const uint32_t* blk_segs;     // segments of each block in tile order
  int nblocks;
};

// Metadata blob of a tile (every section starts on a 16 B boundary):
//   u32 header[4] = {nobs, npt, nseg, seg_base}
//   u32 w0[nobs]      pose parameter offset | pose dim << 28
//   u32 w1[nobs]      intrinsic parameter offset | intrinsic dim << 28
//   u16 lpt[nobs]     local point of the observation
//   u16 poff[npt+1]   local observation range of each point
//   u32 sg[nseg]      block parameter offset | block dim << 28
//   u16 segb[nseg+1]  entity range of each segment
//   u16 ent[nent]     local observation | column code << 12 (0: column 0, 1: 5, 2: 6)
struct BlobView {
  uint32_t nobs, npt, nseg, seg_base;
  const uint32_t* w0;
  const uint32_t* w1;
  const uint16_t* lpt;
  const uint16_t* poff;
  const uint32_t* sg;
  const uint16_t* segb;
  const uint16_t* ent;
};
__host__ __device__ __forceinline__ size_t align16(size_t x) { return (x + 15) & ~size_t(15); }
// Section offsets of a blob with the given counts; returns the total (16 B multiple) size.
__host__ __device__ __forceinline__ size_t blob_layout(uint32_t nobs, uint32_t npt, uint32_t nseg, uint32_t nent,
                                                      size_t off[7]) {
  size_t o = 16;
  off[0] = o;
  o = align16(o + 4 * (size_t)nobs);
  off[1] = o;
  o = align16(o + 4 * (size_t)nobs);
  off[2] = o;
  o = align16(o + 2 * (size_t)nobs);
  off[3] = o;
  o = align16(o + 2 * (size_t)(npt + 1));
  off[4] = o;
  o = align16(o + 4 * (size_t)nseg);
  off[5] = o;
  o = align16(o + 2 * (size_t)(nseg + 1));
  off[6] = o;
  o = align16(o + 2 * (size_t)nent);
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
  blob_layout(v.nobs, v.npt, v.nseg, 0, off);
  v.w0 = reinterpret_cast<const uint32_t*>(b + off[0]);
  v.w1 = reinterpret_cast<const uint32_t*>(b + off[1]);
  v.lpt = reinterpret_cast<const uint16_t*>(b + off[2]);
  v.poff = reinterpret_cast<const uint16_t*>(b + off[3]);
  v.sg = reinterpret_cast<const uint32_t*>(b + off[4]);
  v.segb = reinterpret_cast<const uint16_t*>(b + off[5]);
  v.ent = reinterpret_cast<const uint16_t*>(b + off[6]);
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

template <typename T>
__host__ __device__ constexpr int mv_tile_obs() {
  return sizeof(T) == 4 ? 256 : 128;
}
// Upper bound of a tile's metadata blob (nseg <= 2 TILE, nent <= 2 TILE, npt <= TILE).
__host__ __device__ constexpr size_t mv_blob_max(int tile) { return 16 + 28 * (size_t)tile + 8 * 16 + 16; }
template <typename T>
__host__ __device__ constexpr size_t mv_stage_bytes() {
  return align16(sizeof(T) * (size_t)mv_tile_obs<T>() * kRec) + align16(mv_blob_max(mv_tile_obs<T>())) +
         48 * (size_t)mv_tile_obs<T>();
}
// Records of a tile live at rec + t * TILE * kRec; a partial tile's unused slots are zero.
template <typename T>
__host__ __device__ constexpr size_t mv_smem_bytes() {
  // two stages, plus e/f (2 per observation), point terms (3 per observation), z (3 per point)
  return 2 * mv_stage_bytes<T>() + sizeof(T) * (size_t)mv_tile_obs<T>() * 8;
}

__device__ __forceinline__ int colcode_to_col(int code) { return code == 0 ? 0 : (code == 1 ? 5 : 6); }

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
__global__ void __launch_bounds__(256) k_mv_tiles(MvTiles mt, const T* __restrict__ rec,
                                                  const double* __restrict__ vinv, const double* __restrict__ x,
                                                  double* __restrict__ partial, const PcgCtl* ctl, int* fault) {
  if (pcg_stopped(ctl)) return;
  constexpr int TILE = mv_tile_obs<T>();
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* stage_ptr[2] = {smem_raw, smem_raw + mv_stage_bytes<T>()};
  T* f0 = reinterpret_cast<T*>(smem_raw + 2 * mv_stage_bytes<T>());
  T* f1 = f0 + TILE;
  T* tb = f1 + TILE;
  T* zz = tb + 3 * TILE;
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
  if (t < mt.ntiles && tid == 0) mv_issue_tile<T>(mt, t, rec, vinv, stage_ptr[0], &bar[0]);
  for (int k = 0; t < mt.ntiles; t += gridDim.x, ++k) {
    const int stage = k & 1;
    const int tn = t + gridDim.x;
    bool issued_next = false;
    if (tid == 0 && tn < mt.ntiles) {
      // the other stage was last read by the previous tile; order those reads before the async writes
      fence_proxy_async();
      mv_issue_tile<T>(mt, tn, rec, vinv, stage_ptr[stage ^ 1], &bar[stage ^ 1]);
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
    const T* cur = reinterpret_cast<const T*>(stage_ptr[stage]);
    const BlobView bv = blob_view(stage_ptr[stage] + align16(sizeof(T) * (size_t)TILE * kRec));
    const double* vi_s = reinterpret_cast<const double*>(stage_ptr[stage] + align16(sizeof(T) * (size_t)TILE * kRec) +
                                                         align16(mv_blob_max(TILE)));
    const uint32_t nobs = bv.nobs, npt = bv.npt, nseg = bv.nseg;
    // e_o = Jc_o x_o and the point terms Jp_o^T e_o (component k of observation i at k * TILE + i)
    for (uint32_t i = tid; i < nobs; i += blockDim.x) {
      const T* r = cur + i;
      const uint32_t w0 = bv.w0[i], w1 = bv.w1[i];
      const int pd = (int)(w0 >> 28), id = (int)(w1 >> 28);
      const uint32_t po = w0 & 0x0FFFFFFFu, io = w1 & 0x0FFFFFFFu;
      T e0 = 0, e1 = 0;
      for (int c = 0; c < pd; ++c) {
        T xv = (T)__ldg(x + po + c);
        e0 += r[c * TILE] * xv;
        e1 += r[(9 + c) * TILE] * xv;
      }
      for (int c = 0; c < id; ++c) {
        T xv = (T)__ldg(x + io + c);
        e0 += r[(pd + c) * TILE] * xv;
        e1 += r[(9 + pd + c) * TILE] * xv;
      }
      f0[i] = e0;
      f1[i] = e1;
      const T* jp = r + kJp * TILE;
      tb[3 * i] = jp[0] * e0 + jp[3 * TILE] * e1;
      tb[3 * i + 1] = jp[TILE] * e0 + jp[4 * TILE] * e1;
      tb[3 * i + 2] = jp[2 * TILE] * e0 + jp[5 * TILE] * e1;
    }
    __syncthreads();
    // z_p = Vhat_p^-1 sum_o Jp_o^T e_o (sequential per point: fixed order)
    for (uint32_t lp = tid; lp < npt; lp += blockDim.x) {
      const uint32_t a = bv.poff[lp], b = bv.poff[lp + 1];
      T b0 = 0, b1 = 0, b2 = 0;
      for (uint32_t i = a; i < b; ++i) {
        b0 += tb[3 * i];
        b1 += tb[3 * i + 1];
        b2 += tb[3 * i + 2];
      }
      const double* vi = vi_s + 6 * (size_t)lp;
      const T v0 = (T)vi[0], v1 = (T)vi[1], v2 = (T)vi[2], v3 = (T)vi[3], v4 = (T)vi[4], v5 = (T)vi[5];
      zz[3 * lp] = v0 * b0 + v1 * b1 + v3 * b2;
      zz[3 * lp + 1] = v1 * b0 + v2 * b1 + v4 * b2;
      zz[3 * lp + 2] = v3 * b0 + v4 * b1 + v5 * b2;
    }
    __syncthreads();
    // f_o = e_o - Jp_o z_p
    for (uint32_t i = tid; i < nobs; i += blockDim.x) {
      const int lp = bv.lpt[i];
      const T* jp = cur + kJp * TILE + i;
      const T z0 = zz[3 * lp], z1 = zz[3 * lp + 1], z2 = zz[3 * lp + 2];
      f0[i] -= jp[0] * z0 + jp[TILE] * z1 + jp[2 * TILE] * z2;
      f1[i] -= jp[3 * TILE] * z0 + jp[4 * TILE] * z1 + jp[5 * TILE] * z2;
    }
    __syncthreads();
    // one thread per (segment, component): partial_c = sum_e (Jc_e^T f_o)_c in entity order
    for (uint32_t w = tid; w < 6 * nseg; w += blockDim.x) {
      const uint32_t s = w / 6, c = w - 6 * s;
      const int d = (int)(bv.sg[s] >> 28);
      if ((int)c >= d) continue;
      T acc = 0;
      for (uint32_t j = bv.segb[s]; j < bv.segb[s + 1]; ++j) {
        const uint16_t e = bv.ent[j];
        const int li = e & 0x0fff, col = colcode_to_col(e >> 12);
        acc += cur[(col + c) * TILE + li] * f0[li] + cur[(9 + col + c) * TILE + li] * f1[li];
      }
      partial[6 * (size_t)(bv.seg_base + s) + c] = (double)acc;
    }
    __syncthreads();
  }
}

// y_b = sum over the block's segments + lambda * diag_b * x_b; one warp per block, lane l sums
// segments l, l+32, ... in tile order, then a fixed shuffle tree: deterministic.
__global__ void k_mv_tiles_finalize(MvTiles mt, const double* partial, const double* diag, double lambda,
                                    const double* x, double* y, const PcgCtl* ctl) {
  if (pcg_stopped(ctl)) return;
  int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (b >= mt.nblocks) return;
  int o = mt.blk_off[b], d = mt.blk_dim[b];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (uint32_t i = mt.blk_seg_off[b] + lane; i < mt.blk_seg_off[b + 1]; i += 32) {
    const double* pp = partial + 6 * (size_t)mt.blk_segs[i];
#pragma unroll
    for (int c = 0; c < 6; ++c)
      if (c < d) acc[c] += pp[c];
  }
#pragma unroll
  for (int c = 0; c < 6; ++c) acc[c] = warp_sum(acc[c]);  // full sums land in lane 0
  if (lane == 0)
    for (int c = 0; c < d; ++c) y[o + c] = acc[c] + lambda * diag[o + c] * x[o + c];
}

}  // namespace omvgba
