// mv_tiles.cuh — matrix-free reduced-camera-system product y = S_lambda x for the PCG loop.
//
// S x = sum_o Jc_o^T (e_o - Jp_o z_p) + lambda diag x, with e_o = Jc_o x and
// z_p = Vhat_p^-1 sum_o Jp_o^T e_o (retained/operator.rs:137-227 computes the same product from
// cached Vhat^-1 W^T rows).
//
// Layout: observations are point-major; a tile is a run of whole points with at most TILE
// observations, and one CTA of TILE threads computes one tile, one observation per thread. The
// tile's Jacobian records are component-major (component k of observation i at k TILE + i), so
// each of a thread's 24 record loads is one coalesced line per warp, straight into registers; the
// tile's metadata sits in a fixed-size slot, so every address a CTA needs first is known at launch
// and those loads issue together. Shared memory holds only the small per-tile term arrays, so
// several CTAs share an SM and hide each other's load latency; each CTA also prefetches into L2 the
// records of the tile one resident wave ahead.
//
// Per tile, with a (tile, camera) "segment" for each camera the tile's observations see:
//   P0  x of each segment's pose and intrinsic parameters into shared memory (one gather per
//       segment and parameter instead of one per observation);
//   P1  thread per observation: e = Jc x, point terms Jp^T e;
//   P2  four lanes per point (one per component of the track sum, in track order, exchanged by
//       shuffles): z = Vhat^-1 (sum of the point terms);
//   P3  thread per observation: f = e - Jp z and its camera terms Jc^T f, stored in segment order;
//   P4  thread per (segment, parameter): the sum of the segment's contiguous run of camera terms,
//       in observation order, written to the segment's place in its block's partial region.
// The finalize kernel sums each block's contiguous partial region in tile order (one warp per
// block, fixed lane assignment and shuffle tree) and adds lambda diag x. No sum depends on
// scheduling, so the product is bitwise reproducible run to run.
#pragma once

#include <cstdint>

namespace omvgba {

template <typename T>
__host__ __device__ constexpr int mv_tile_obs() {
  return sizeof(T) == 4 ? 256 : 128;
}
constexpr int kSegParams = 9;  // pose (<= 6) then intrinsic (<= 3) parameters of a segment
constexpr uint32_t kNoPartial = 0xFFFFFFFFu;

// Fixed-size metadata slot of a tile with TILE observations (byte offsets):
//   u32 w0[TILE]        pose parameter offset | pose dim << 28, per segment
//   u32 w1[TILE]        intrinsic parameter offset | intrinsic dim << 28, per segment
//   u32 dpose[TILE]     first partial of the segment's pose part (kNoPartial: none), per segment
//   u32 dintr[TILE]     first partial of the segment's intrinsic part (kNoPartial: none)
//   u16 segb[TILE + 1]  range of each segment in segment order (padded to 16 B)
//   u16 oseg[TILE]      segment of each observation
//   u16 lpt[TILE]       local point of each observation
//   u16 pos[TILE]       position of each observation in segment order
//   u16 poff[TILE + 1]  local observation range of each point (padded to 16 B)
struct MvSlot {
  static constexpr size_t w0(int) { return 0; }
  static constexpr size_t w1(int tile) { return 4 * (size_t)tile; }
  static constexpr size_t dpose(int tile) { return 8 * (size_t)tile; }
  static constexpr size_t dintr(int tile) { return 12 * (size_t)tile; }
  static constexpr size_t segb(int tile) { return 16 * (size_t)tile; }
  static constexpr size_t oseg(int tile) { return 18 * (size_t)tile + 16; }
  static constexpr size_t lpt(int tile) { return 20 * (size_t)tile + 16; }
  static constexpr size_t pos(int tile) { return 22 * (size_t)tile + 16; }
  static constexpr size_t poff(int tile) { return 24 * (size_t)tile + 16; }
  static constexpr size_t bytes(int tile) { return (26 * (size_t)tile + 32 + 127) & ~size_t(127); }
};

struct MvTiles {
  int ntiles;
  const uint4* tile_hdr;       // per tile: {observations, points, segments, first point}
  const unsigned char* slots;  // per tile: MvSlot::bytes(TILE)
  int nblocks;
  const int* blk_dim;
  const int* blk_off;
  const uint32_t* blk_part;    // nblocks + 1: each block's partial region (segment-major, dim wide)
  int prefetch_ahead;          // tiles ahead (about one resident wave) whose records are prefetched
};

// The records are read once per product and are larger than L2; an evict-first policy on their
// prefetch and loads keeps the data that every product re-reads (slots, point blocks, x) resident.
// The bulk prefetch into L2 is a hint (nothing waits for it); bytes % 16 == 0.
__device__ __forceinline__ uint64_t l2_evict_first() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ void bulk_prefetch_l2_hint(const void* src, uint32_t bytes, uint64_t pol) {
  asm volatile("cp.async.bulk.prefetch.L2.global.L2::cache_hint [%0], %1, %2;" ::"l"(src), "r"(bytes), "l"(pol)
               : "memory");
}
__device__ __forceinline__ float ld_stream(const float* p, uint64_t pol) {
  float v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ double ld_stream(const double* p, uint64_t pol) {
  double v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}

// R: the records' storage type (it sets the tile size); T: the arithmetic type (T = double with
// R = float is the FP64 product of FP32-stored Jacobians that mixed-precision refinement uses).
template <typename R, typename T = R>
__global__ void __launch_bounds__(mv_tile_obs<R>(), sizeof(T) == sizeof(R) ? 4 : 2)
    k_mv_tiles(MvTiles mt, const R* __restrict__ rec, const double* __restrict__ vfac, const double* __restrict__ x,
               double* __restrict__ partial, const PcgCtl* ctl) {
  constexpr int TILE = mv_tile_obs<R>();
  constexpr int TS = TILE + 1;  // padded row stride: the 9 parameter rows of one column use 9 banks
  __shared__ T xs[kSegParams * TILE];
  __shared__ T zz[3 * TILE];
  __shared__ T terms[kSegParams * TS];
  __shared__ uint4 seg_info[TILE];        // w0, w1, dpose, dintr per segment
  __shared__ uint16_t seg_begin[TILE + 1];
  __shared__ uint16_t pt_begin[TILE + 1];
  const int t = blockIdx.x, tid = threadIdx.x;
  // Within one graph launch a PCG run that has stopped stays stopped (the host resets the control
  // block only between launches), so a stop seen before the wait is final: the iterations enqueued
  // past the end of the run then skip their record loads too, not just their arithmetic.
  if (ctl && *reinterpret_cast<const volatile int*>(&ctl->status) != kRunning) return;
  // The CTA that starts about one resident wave later finds its records in L2.
  const uint64_t stream_pol = l2_evict_first();
  if (tid == 0 && mt.prefetch_ahead > 0 && t + mt.prefetch_ahead < mt.ntiles)
    bulk_prefetch_l2_hint(rec + (size_t)(t + mt.prefetch_ahead) * TILE * kRec, (uint32_t)(sizeof(R) * TILE * kRec),
                          stream_pol);
  // Every first load depends only on (t, tid), so they all issue together: the records, the header
  // and one entry of each slot column (thread s loads segment s's row; rows past the tile's
  // segment count are zero).
  const R* r = rec + (size_t)t * TILE * kRec + tid;  // a partial tile's unused records are zero
  T jc[18], jp[6];
#pragma unroll
  for (int c = 0; c < 18; ++c) jc[c] = (T)ld_stream(r + c * TILE, stream_pol);
#pragma unroll
  for (int c = 0; c < 6; ++c) jp[c] = (T)ld_stream(r + (kJp + c) * TILE, stream_pol);
  const uint4 hdr = mt.tile_hdr[t];
  const unsigned char* slot = mt.slots + (size_t)t * MvSlot::bytes(TILE);
  const uint32_t my_w0 = __ldg(reinterpret_cast<const uint32_t*>(slot + MvSlot::w0(TILE)) + tid);
  const uint32_t my_w1 = __ldg(reinterpret_cast<const uint32_t*>(slot + MvSlot::w1(TILE)) + tid);
  const uint32_t my_dpose = __ldg(reinterpret_cast<const uint32_t*>(slot + MvSlot::dpose(TILE)) + tid);
  const uint32_t my_dintr = __ldg(reinterpret_cast<const uint32_t*>(slot + MvSlot::dintr(TILE)) + tid);
  const uint16_t* segb = reinterpret_cast<const uint16_t*>(slot + MvSlot::segb(TILE));
  const uint16_t* poff = reinterpret_cast<const uint16_t*>(slot + MvSlot::poff(TILE));
  const uint16_t my_segb = __ldg(segb + tid), my_poff = __ldg(poff + tid);
  const uint32_t my_seg = __ldg(reinterpret_cast<const uint16_t*>(slot + MvSlot::oseg(TILE)) + tid);
  const uint32_t my_pt = __ldg(reinterpret_cast<const uint16_t*>(slot + MvSlot::lpt(TILE)) + tid);
  const uint32_t my_pos = __ldg(reinterpret_cast<const uint16_t*>(slot + MvSlot::pos(TILE)) + tid);
  const uint32_t nobs = hdr.x, npt = hdr.y, nseg = hdr.z, p0 = hdr.w;
  // P2's factor entries for the first TILE / 4 points, requested as soon as the header is in. Lane
  // kq of a point's quad loads entries i0, i1, i2 of the packed lower factor N (Vhat^-1 = N^T N):
  // row kq of N is (v0, 0, 0), (v0, v1, 0), (v0, v1, v2) and column kq is (v0, v1, v2), (0, v1, v2),
  // (0, 0, v2) for kq = 0, 1, 2.
  const uint32_t lp0 = tid >> 2, kq = tid & 3;
  const int i0 = kq == 0 ? 0 : (kq == 1 ? 1 : 3), i1 = kq == 0 ? 1 : (kq == 1 ? 2 : 4), i2 = kq == 0 ? 3 : (kq == 1 ? 4 : 5);
  double v0 = 0.0, v1 = 0.0, v2 = 0.0;
  if (lp0 < npt && kq < 3) {
    const double* vi = vfac + 6 * (size_t)(p0 + lp0);
    v0 = __ldg(vi + i0);
    v1 = __ldg(vi + i1);
    v2 = __ldg(vi + i2);
  }
  // Everything above is constant during the PCG loop; x and the control block come from the kernels
  // before this one.
  pdl_trigger();
  pdl_wait();
  if (pcg_stopped(ctl)) return;
  // P0: thread s gathers x for segment s's parameters (zero beyond its dimensions) and stages the
  // segment's row, the segment ranges and the point ranges in shared memory
  {
    const uint32_t pd = my_w0 >> 28, id = my_w1 >> 28;
    T xv[kSegParams];
#pragma unroll
    for (int c = 0; c < kSegParams; ++c) {
      // one predicated load per column (pose columns, then intrinsic columns, then zeros)
      const uint32_t at = (uint32_t)c < pd ? (my_w0 & 0x0FFFFFFFu) + c : (my_w1 & 0x0FFFFFFFu) + ((uint32_t)c - pd);
      const double v = (uint32_t)c < pd + id ? __ldg(x + at) : 0.0;
      xv[c] = (T)v;
    }
    if ((uint32_t)tid < nseg) {
#pragma unroll
      for (int c = 0; c < kSegParams; ++c) xs[kSegParams * tid + c] = xv[c];
    }
    seg_info[tid] = make_uint4(my_w0, my_w1, my_dpose, my_dintr);
    seg_begin[tid] = my_segb;
    pt_begin[tid] = my_poff;
    if (tid == 0) {
      seg_begin[TILE] = __ldg(segb + TILE);
      pt_begin[TILE] = __ldg(poff + TILE);
    }
  }
  __syncthreads();
  // P1: e = Jc x (two accumulators per row: shorter dependency chains) and the point terms Jp^T e
  T e0 = 0, e1 = 0;
  if ((uint32_t)tid < nobs) {
    const T* xv = xs + kSegParams * my_seg;
    T e0b = 0, e1b = 0;
#pragma unroll
    for (int c = 0; c < 9; c += 2) {
      e0 += jc[c] * xv[c];
      e1 += jc[9 + c] * xv[c];
    }
#pragma unroll
    for (int c = 1; c < 9; c += 2) {
      e0b += jc[c] * xv[c];
      e1b += jc[9 + c] * xv[c];
    }
    e0 += e0b;
    e1 += e1b;
    terms[tid] = jp[0] * e0 + jp[3] * e1;
    terms[TS + tid] = jp[1] * e0 + jp[4] * e1;
    terms[2 * TS + tid] = jp[2] * e0 + jp[5] * e1;
  }
  __syncthreads();
  // P2: z_p = Vhat_p^-1 sum_o Jp_o^T e_o = N^T (N b); lanes 4q..4q+2 of a warp sum the three
  // components of point q's track (in track order), lane 4q+3 idles; b and then u = N b are exchanged
  // by shuffles.
  for (uint32_t base = 0; base < npt; base += TILE / 4) {
    const uint32_t lp = base + lp0;
    const bool active = lp < npt && kq < 3;
    T bk = 0;
    if (active) {
      const T* row = terms + kq * TS;
      const uint32_t e = pt_begin[lp + 1];
      for (uint32_t i = pt_begin[lp]; i < e; ++i) bk += row[i];
      if (base > 0) {  // points past the first TILE / 4: their factor entries load here
        const double* vi = vfac + 6 * (size_t)(p0 + lp);
        v0 = __ldg(vi + i0);
        v1 = __ldg(vi + i1);
        v2 = __ldg(vi + i2);
      }
    }
    const int lead = (tid & 31) & ~3;
    const T b0 = __shfl_sync(0xffffffffu, bk, lead), b1 = __shfl_sync(0xffffffffu, bk, lead + 1),
            b2 = __shfl_sync(0xffffffffu, bk, lead + 2);
    const T n0 = (T)v0, n1 = (T)v1, n2 = (T)v2;
    const T uk = n0 * b0 + (kq >= 1 ? n1 * b1 : (T)0) + (kq == 2 ? n2 * b2 : (T)0);  // (N b)_kq
    const T u0 = __shfl_sync(0xffffffffu, uk, lead), u1 = __shfl_sync(0xffffffffu, uk, lead + 1),
            u2 = __shfl_sync(0xffffffffu, uk, lead + 2);
    if (active) zz[kq * TILE + lp] = (kq == 0 ? n0 * u0 : (T)0) + (kq <= 1 ? n1 * u1 : (T)0) + n2 * u2;
  }
  __syncthreads();
  // P3: f = e - Jp z and the camera terms Jc^T f in segment order (the point terms are dead)
  if ((uint32_t)tid < nobs) {
    const T z0 = zz[my_pt], z1 = zz[TILE + my_pt], z2 = zz[2 * TILE + my_pt];
    const T f0 = e0 - (jp[0] * z0 + jp[1] * z1 + jp[2] * z2);
    const T f1 = e1 - (jp[3] * z0 + jp[4] * z1 + jp[5] * z2);
#pragma unroll
    for (int c = 0; c < 9; ++c) terms[c * TS + my_pos] = jc[c] * f0 + jc[9 + c] * f1;
  }
  __syncthreads();
  // P4: per (segment, parameter) sum of the segment's run of camera terms in observation order
  for (uint32_t w = tid; w < kSegParams * nseg; w += TILE) {
    const uint32_t s = w / kSegParams, c = w - kSegParams * s;
    const uint4 si = seg_info[s];
    const uint32_t pd = si.x >> 28, id = si.y >> 28;
    if (c >= pd + id) continue;
    T acc = 0;
    const T* col = terms + c * TS;
    const uint32_t e = seg_begin[s + 1];
    for (uint32_t q = seg_begin[s]; q < e; ++q) acc += col[q];
    partial[c < pd ? si.z + c : si.w + (c - pd)] = (double)acc;
  }
}

// y_b = sum of block b's partials (its segments in tile order) + lambda diag_b x_b: one warp per
// block; lane l sums segments l, l + 32, ... of the block's contiguous region in order, then a
// fixed shuffle tree. A block no observation touches has an empty region: y_b = lambda diag_b x_b.
// With xy non-null, xy[CTA] = sum over the CTA's blocks, in block order, of x_b . y_b (the PCG
// curvature terms).
__global__ void __launch_bounds__(256) k_mv_tiles_finalize(MvTiles mt, const double* __restrict__ partial,
                                                           const double* __restrict__ diag, double lambda,
                                                           const double* __restrict__ x, double* __restrict__ y,
                                                           double* __restrict__ xy, const PcgCtl* ctl) {
  __shared__ double s_dot[8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = blockIdx.x * 8 + warp;
  // the block's layout and diagonal are constant during the PCG loop: loaded before the wait
  const bool have = b < mt.nblocks;
  const int o = have ? mt.blk_off[b] : 0, d = have ? mt.blk_dim[b] : 0;
  const uint32_t a0 = have ? mt.blk_part[b] : 0u, a1 = have ? mt.blk_part[b + 1] : 0u;
  double dg[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) dg[c] = lane == 0 && c < d ? diag[o + c] : 0.0;
  pdl_trigger();
  pdl_wait();
  if (pcg_stopped(ctl)) return;
  double dot = 0.0;
  if (have) {
    double xv[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) xv[c] = lane == 0 && c < d ? x[o + c] : 0.0;
    const uint32_t nseg = d > 0 ? (a1 - a0) / (uint32_t)d : 0u;
    double acc[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll 4
    for (uint32_t j = lane; j < nseg; j += 32) {
      const double* pp = partial + a0 + (size_t)j * d;
#pragma unroll
      for (int c = 0; c < 6; ++c)
        if (c < d) acc[c] += pp[c];
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) acc[c] = warp_sum(acc[c]);  // full sums land in lane 0
    if (lane == 0) {
#pragma unroll
      for (int c = 0; c < 6; ++c)
        if (c < d) {
          const double v = acc[c] + lambda * dg[c] * xv[c];
          y[o + c] = v;
          dot += xv[c] * v;
        }
    }
  }
  if (xy) {
    if (lane == 0) s_dot[warp] = dot;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < 8; ++w) t += s_dot[w];
      xy[blockIdx.x] = t;
    }
  }
}

}  // namespace omvgba
