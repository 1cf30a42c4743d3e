// asm_tiles.cuh — the camera-side assembly (schur/assembly.rs:893-1069: U blocks, g, the reduced g,
// the damping diagonal, the pose/intrinsic edges and the point coupling of each block's diagonal)
// as a pass over the tiles of the Jacobian records, then a per-block sum.
//
// k_block_tiles: one CTA per tile, one thread per observation, reading the component-major records
// coalesced. Each thread stages its observation's camera columns, residuals and point coupling in
// shared memory, in segment order; then each thread takes one (segment, block row) — a row of the
// segment's pose block or of its intrinsic group's block — and sums that row's terms over the
// segment's observations in order. The sums land in the segment's record of each block: the records
// of block b follow its matrix-free partial region (blk_part) at 12 doubles per partial element, in
// tile order. k_block_records then sums each block's records in that order into the assembly record
// (kAsmRec) the preconditioner and the vectors read. Every sum runs in a fixed order.
//
// Record of a block of dimension d (T = d (d + 1) / 2; lower triangles packed by r (r + 1) / 2 + s):
//   U [T] | g [d] | reduced g [d] | coupling [T] | edge [3 d] (pose blocks: U of pose row r and
//   intrinsic column k at 3 r + k)
#pragma once

namespace omvgba {

constexpr int kAsmRecordScale = 12;  // doubles of a block record per element of its partial region
// Staged components of an observation (rows of the shared table, one column per observation in
// segment order): the two residual rows' 9 camera columns, weighted residual and reduced residual at
// 0..10 and 11..21 (row 1 = row 0 + kAsmRow1), then A = Jp Vhat^-1 Jp^T (A00, A01, A11).
constexpr int kAsmRow1 = 11;
constexpr int kAsmComp = 25;
constexpr int kAsmRes = 9, kAsmRed = 10, kAsmA = 22;

// offset of a term in a block record of dimension d: kind 0 U, 1 g, 2 reduced g, 3 coupling, 4 edge
__device__ __forceinline__ int asm_offset(int d, int kind, int r, int s) {
  const int T = d * (d + 1) / 2;
  switch (kind) {
    case 0: return r * (r + 1) / 2 + s;
    case 1: return T + r;
    case 2: return T + d + r;
    case 3: return T + 2 * d + r * (r + 1) / 2 + s;
    default: return 2 * T + 2 * d + 3 * r + s;
  }
}

template <typename R>
constexpr int asm_min_blocks() {
  return 3 * 256 / mv_tile_obs<R>();
}
template <typename R>
constexpr size_t asm_smem_bytes() {
  return sizeof(double) * kAsmComp * (mv_tile_obs<R>() + 1);
}

template <typename R>
__global__ void __launch_bounds__(mv_tile_obs<R>(), asm_min_blocks<R>())
    k_block_tiles(MvTiles mt, LinOut<R> lin, const uint32_t* __restrict__ pt_off, double* __restrict__ rec_out) {
  constexpr int TILE = mv_tile_obs<R>();
  constexpr int TS = TILE + 1;
  extern __shared__ double D[];     // kAsmComp x TS
  __shared__ uint4 seg_info[TILE];  // w0, w1, pose record, intrinsic record per segment
  __shared__ uint16_t seg_begin[TILE + 1];
  const int t = blockIdx.x, tid = threadIdx.x;
  const uint4 hdr = mt.tile_hdr[t];
  const unsigned char* slot = mt.slots + (size_t)t * MvSlot::bytes(TILE);
  const uint32_t* w0 = reinterpret_cast<const uint32_t*>(slot + MvSlot::w0(TILE));
  const uint32_t* w1 = reinterpret_cast<const uint32_t*>(slot + MvSlot::w1(TILE));
  const uint16_t* segb = reinterpret_cast<const uint16_t*>(slot + MvSlot::segb(TILE));
  const uint32_t nobs = hdr.x, nseg = hdr.z, p0 = hdr.w;
  seg_info[tid] = make_uint4(w0[tid], w1[tid], reinterpret_cast<const uint32_t*>(slot + MvSlot::dpose(TILE))[tid],
                             reinterpret_cast<const uint32_t*>(slot + MvSlot::dintr(TILE))[tid]);
  seg_begin[tid] = segb[tid];
  if (tid == 0) seg_begin[TILE] = segb[TILE];
  // this observation's columns, residual, reduced residual r_w - Jp (Vhat^-1 g_p) and point
  // coupling A, as schur/assembly.rs:893-1069 forms them
  if ((uint32_t)tid < nobs) {
    const R* rr = lin.rec + (size_t)t * TILE * kRec + tid;
    const uint32_t pos = reinterpret_cast<const uint16_t*>(slot + MvSlot::pos(TILE))[tid];
    double* col = D + pos;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      col[c * TS] = (double)rr[(size_t)c * TILE];
      col[(kAsmRow1 + c) * TS] = (double)rr[(size_t)(9 + c) * TILE];
    }
    const double pv0[3] = {(double)rr[(size_t)kJp * TILE], (double)rr[(size_t)(kJp + 1) * TILE],
                           (double)rr[(size_t)(kJp + 2) * TILE]};
    const double pv1[3] = {(double)rr[(size_t)(kJp + 3) * TILE], (double)rr[(size_t)(kJp + 4) * TILE],
                           (double)rr[(size_t)(kJp + 5) * TILE]};
    const uint32_t lp = reinterpret_cast<const uint16_t*>(slot + MvSlot::lpt(TILE))[tid];
    const size_t o = (size_t)pt_off[p0] + tid, p = (size_t)p0 + lp;
    const double r0 = lin.rw[2 * o], r1 = lin.rw[2 * o + 1];
    const double* ig = lin.ig + 3 * p;
    col[kAsmRes * TS] = r0;
    col[(kAsmRow1 + kAsmRes) * TS] = r1;
    col[kAsmRed * TS] = r0 - (pv0[0] * ig[0] + pv0[1] * ig[1] + pv0[2] * ig[2]);
    col[(kAsmRow1 + kAsmRed) * TS] = r1 - (pv1[0] * ig[0] + pv1[1] * ig[1] + pv1[2] * ig[2]);
    double t0[3], t1[3];
    sym3_apply(lin.vinv + 6 * p, pv0, t0);
    sym3_apply(lin.vinv + 6 * p, pv1, t1);
    col[kAsmA * TS] = pv0[0] * t0[0] + pv0[1] * t0[1] + pv0[2] * t0[2];
    col[(kAsmA + 1) * TS] = pv0[0] * t1[0] + pv0[1] * t1[1] + pv0[2] * t1[2];
    col[(kAsmA + 2) * TS] = pv1[0] * t1[0] + pv1[1] * t1[1] + pv1[2] * t1[2];
  }
  __syncthreads();
  // one (segment, block row) per thread: row r of the segment's pose block (0..5) or intrinsic
  // block (6..8) with U(r, s <= r), the coupling (r, s <= r), g, the reduced g and, for pose rows,
  // the edge to the segment's intrinsic columns, each summed over the segment in order
  for (uint32_t w = tid; w < nseg * (uint32_t)kSegParams; w += TILE) {
    const uint32_t sg = w / kSegParams;
    const int row = (int)(w - sg * kSegParams);
    const uint4 si = seg_info[sg];
    const int pd = (int)(si.x >> 28), id = (int)(si.y >> 28);
    const bool pose = row < 6;
    const int r = pose ? row : row - 6, d = pose ? pd : id;
    const uint32_t base = pose ? si.z : si.w;
    if (base == kNoPartial || r >= d) continue;
    const int cb = pose ? 0 : pd;    // the block's first column among the 9
    const int ne = pose ? id : 0;    // edge columns
    double u[6], cp[6], e[3], g = 0.0, gq = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) u[k] = cp[k] = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) e[k] = 0.0;
    const double* X = D + (cb + r) * TS;
    for (uint32_t q = seg_begin[sg]; q < seg_begin[sg + 1]; ++q) {
      const double x0 = X[q], x1 = X[kAsmRow1 * TS + q];
      const double A00 = D[kAsmA * TS + q], A01 = D[(kAsmA + 1) * TS + q], A11 = D[(kAsmA + 2) * TS + q];
      const double c0 = x0 * A00 + x1 * A01, c1 = x0 * A01 + x1 * A11;
      g += x0 * D[kAsmRes * TS + q] + x1 * D[(kAsmRow1 + kAsmRes) * TS + q];
      gq += x0 * D[kAsmRed * TS + q] + x1 * D[(kAsmRow1 + kAsmRed) * TS + q];
#pragma unroll
      for (int s2 = 0; s2 < 6; ++s2)
        if (s2 <= r) {
          const double y0 = D[(cb + s2) * TS + q], y1 = D[(kAsmRow1 + cb + s2) * TS + q];
          u[s2] += x0 * y0 + x1 * y1;
          cp[s2] += c0 * y0 + c1 * y1;
        }
#pragma unroll
      for (int k = 0; k < 3; ++k)
        if (k < ne) e[k] += x0 * D[(pd + k) * TS + q] + x1 * D[(kAsmRow1 + pd + k) * TS + q];
    }
    double* out = rec_out + (size_t)base * kAsmRecordScale;
    const int T = d * (d + 1) / 2, tri = r * (r + 1) / 2;
#pragma unroll
    for (int s2 = 0; s2 < 6; ++s2)
      if (s2 <= r) {
        out[tri + s2] = u[s2];
        out[T + 2 * d + tri + s2] = cp[s2];
      }
    out[T + r] = g;
    out[T + d + r] = gq;
#pragma unroll
    for (int k = 0; k < 3; ++k)
      if (k < ne) out[2 * T + 2 * d + 3 * r + k] = e[k];
  }
}

// Per block: the sum of its records in tile order, in the assembly record layout (kAsmRec): U lower
// (21, packed as six rows), g (6), reduced g (6), damping diagonal (6: the diagonal of U), edge (18),
// coupling lower (21); entries past the block's dimension are zero. One CTA per block.
__global__ void __launch_bounds__(128) k_block_records(MvTiles mt, const int* __restrict__ blk_edge,
                                                       const double* __restrict__ rec_in, double* __restrict__ blk_out) {
  const int b = blockIdx.x;
  if (b >= mt.nblocks) return;
  const int d = mt.blk_dim[b];
  const uint32_t e0 = mt.blk_part[b], e1 = mt.blk_part[b + 1];
  const uint32_t n = d > 0 ? (e1 - e0) / (uint32_t)d : 0;
  const size_t stride = (size_t)kAsmRecordScale * d;
  const double* base = rec_in + (size_t)e0 * kAsmRecordScale;
  const int di = blk_edge[b] >= 0 ? mt.blk_dim[blk_edge[b]] : 0;  // the edge's intrinsic columns
  for (int k = threadIdx.x; k < kAsmRec; k += blockDim.x) {
    int off = -1;
    if (k < 21) {
      int r = 0;
      while ((r + 1) * (r + 2) / 2 <= k) ++r;
      if (r < d) off = asm_offset(d, 0, r, k - r * (r + 1) / 2);
    } else if (k < 27) {
      if (k - 21 < d) off = asm_offset(d, 1, k - 21, 0);
    } else if (k < 33) {
      if (k - 27 < d) off = asm_offset(d, 2, k - 27, 0);
    } else if (k < 39) {
      const int r = k - 33;
      if (r < d) off = asm_offset(d, 0, r, r);
    } else if (k < 57) {
      const int r = (k - 39) / 3, c = (k - 39) % 3;
      if (r < d && c < di) off = asm_offset(d, 4, r, c);
    } else {
      const int idx = k - 57;
      int r = 0;
      while ((r + 1) * (r + 2) / 2 <= idx) ++r;
      if (r < d) off = asm_offset(d, 3, r, idx - r * (r + 1) / 2);
    }
    double acc = 0.0;
    if (off >= 0)
      for (uint32_t q = 0; q < n; ++q) acc += base[q * stride + off];
    blk_out[(size_t)kAsmRec * b + k] = acc;
  }
}

}  // namespace omvgba
