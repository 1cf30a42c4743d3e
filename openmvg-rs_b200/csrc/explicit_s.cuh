// explicit_s.cuh — the explicit reduced camera system S and its banded tiled FP64 Cholesky factor.
//
// S = U - W Vhat^-1 W^T over the free camera parameters (schur/assembly.rs:832-1069 assembles the same
// matrix into faer's sparse pattern, sparse/direct_assembly.rs:371-687). Here it is built by block
// rows: one CTA per parameter block X computes every block S_XY of its row (all co-visible blocks Y,
// both triangles), walking X's entities in a fixed order and the entities of each entity's point, so
// the row is the same bits run to run and needs no atomics. The rows serve as a block-sparse (BSR)
// operator directly (the PCG product and the model reduction) and are scattered into a banded tiled
// matrix for the factorization.
//
// Factorization. The parameter blocks are permuted so that each camera's pose block is followed by
// the intrinsic blocks it introduces; with cameras in their native order the co-visibility graph of
// a survey is banded, so the factor fits in a band of tiles (64 x 64 FP64, column-major) and a
// right-looking tiled Cholesky (POTRF of the diagonal tile, TRSM of the tiles below it, SYRK/GEMM
// update of the trailing band) never leaves the band. faer's sparse LLT with an AMD ordering
// (numerics/sparse.rs:119-250) factors the same matrix; the factors agree to rounding and the
// positive-definiteness decision is the same away from rounding-level pivots. Every tile update
// runs in a fixed order, so the factor is bitwise reproducible.
//
// Uses of the factor: the direct camera step (sparse/direct.rs:259-288), the camera rank test of the
// final undamped system (sparse/direct.rs:288-455: the spectral test after Jacobi equilibration
// when D <= 2048, a factorization otherwise), and the self-calibration intrinsic marginal
// covariances (sparse/covariance.rs:564-587) from the selected inverse of S inside the band.
#pragma once

#include <cstdint>

namespace omvgba {

// ---- block rows ---------------------------------------------------------------------------------
struct RowTables {
  int nblocks;
  const int* blk_dim;
  const int* blk_off;
  const uint32_t* blk_ent;    // nb + 1: each block's range in ent
  const uint32_t* ent;        // entity list (observation * 2 + segment), block-major
  const uint32_t* ent_point;  // point of each entity (same order)
  const int* seg_col;         // per entity id: column of its segment in the observation's record
  const int* ent_block;       // per entity id: parameter block, -1 when absent
  const uint32_t* pt_off;     // P + 1
  const uint32_t* nbr_begin;  // nb + 1: each block's range in nbr / slot_off
  const int* nbr;             // neighbour blocks of each block (ascending; the block itself included)
  const int* nbr_row;         // block owning each neighbour entry
  const uint64_t* slot_off;   // entries + 1: offset of block S_XY (dX x dY, row-major) in the rows
  uint32_t entries;           // neighbour entries in total
};


// D = A B + C for 8 x 8 FP64 tiles with k = 4 (mma.sync.m8n8k4 f64): each lane passes one element
// of A, one of B and two of C, updated in place.
__device__ __forceinline__ void dmma_m8n8k4(double a, double b, double& c0, double& c1) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ int find_slot(const int* __restrict__ nbr, uint32_t n0, uint32_t n1, int Y) {
  uint32_t lo = n0, hi = n1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (nbr[mid] < Y)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo < n1 && nbr[lo] == Y) ? (int)(lo - n0) : -1;
}

// Row X of S. Each entity e of X (observation o of point p, camera columns cX..cX+dX of its
// record) meets every entity e' of p's track in a block Y (observation k, columns cY..cY+dY):
//   S_XY += [k == o] A_o,X^T A_o,Y - E_e W_k,Y^T,   E_e = A_o,X^T Jp_o Vhat_p^-1 (dX x 3),
//   W_k,Y = A_k,Y^T Jp_k (dY x 3),
// U, the pose/intrinsic edges and the point coupling in one sum (A = the 2 x 9 camera columns and
// Jp the 2 x 3 point columns of a record).
//
// One CTA per row, kRowWarps warps. The row's entities are taken kRowWarps at a time, one per warp:
// the warp computes E of its entity and W of every observation of the track (a chunk of at most
// kRowStage observations per round; longer tracks take several rounds) into shared memory, and the
// slot of each target. After a barrier every warp adds the batch's contributions to the slots it
// owns (slot index mod kRowWarps), entity by entity in batch order and target by target in track
// order, one tensor-pipe product per target. Each element therefore has one writer and a fixed
// summation order: the row is the same bits run to run, without atomics. The row accumulates in
// shared memory when it has at most row_smem doubles (else in place in global memory) and is
// stored once at the end. Each warp fetches the indices of its next entity a batch ahead.
constexpr int kRowWarps = 8;
constexpr int kRowThreads = 32 * kRowWarps;
constexpr int kRowStage = 16;           // track observations per round (2 targets each: 32 lanes)
constexpr int kRowNbr = 1024;           // neighbour lists up to this length sit in shared memory
constexpr int kRowSmemDoubles = 8192;   // rows up to 64 KB accumulate in shared memory
template <typename R>
__global__ void __launch_bounds__(kRowThreads, 2) k_block_rows(RowTables rt, LinOut<R> lin, int row_smem,
                                                               double* __restrict__ rows) {
  extern __shared__ double row_sh[];
  __shared__ int nbr_s[kRowNbr];                       // neighbour blocks
  __shared__ uint32_t ninf_s[kRowNbr];                 // (offset in the row) << 3 | dY
  __shared__ double Wsh[kRowWarps][kRowStage][27];     // W of each chunk observation, 9 x 3 row-major
  __shared__ double Osh[kRowWarps][32];                // the entity's record: A (18), Jp (6), Vhat^-1 (6)
  __shared__ double Esh[kRowWarps][18];                // E (dX x 3)
  __shared__ int tsl[kRowWarps][2 * kRowStage];        // per target: slot or -1
  __shared__ uint32_t tinf[kRowWarps][2 * kRowStage];  // per target: offset << 3 | dY
  __shared__ int tcd[kRowWarps][2 * kRowStage];        // per target: cY | own << 8 | chunk obs << 9
  __shared__ int item_n[kRowWarps], item_cx[kRowWarps];
  const int X = blockIdx.x, tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  if (X >= rt.nblocks) return;
  const int dX = rt.blk_dim[X];
  const uint32_t n0 = rt.nbr_begin[X], n1 = rt.nbr_begin[X + 1], nn = n1 - n0;
  const bool nbr_local = nn <= (uint32_t)kRowNbr;
  const uint64_t r0 = rt.slot_off[n0], r1 = rt.slot_off[n1];
  if (nbr_local)
    for (uint32_t k = tid; k < nn; k += kRowThreads) {
      const int Y = rt.nbr[n0 + k];
      nbr_s[k] = Y;
      ninf_s[k] = (uint32_t)(rt.slot_off[n0 + k] - r0) << 3 | (uint32_t)rt.blk_dim[Y];
    }
  const uint32_t rlen = (uint32_t)(r1 - r0);
  double* row = rlen <= (uint32_t)row_smem ? row_sh : rows + r0;
  for (uint32_t k = tid; k < rlen; k += kRowThreads) row[k] = 0.0;
  const uint32_t i0 = rt.blk_ent[X], i1 = rt.blk_ent[X + 1];
  const int rs = lin.rs;
  // this warp's entity in the current batch (ce, cp, ca = first observation of the track, cl =
  // track length; cl = 0: none) and the next batch's entity and point
  uint32_t ce = 0, cp = 0, ca = 0, cl = 0, xe = 0, xp = 0;
  if (i0 + w < i1) {
    ce = rt.ent[i0 + w];
    cp = rt.ent_point[i0 + w];
    ca = rt.pt_off[cp];
    cl = rt.pt_off[cp + 1] - ca;
  }
  if (i0 + kRowWarps + w < i1) {
    xe = rt.ent[i0 + kRowWarps + w];
    xp = rt.ent_point[i0 + kRowWarps + w];
  }
  for (uint32_t base = i0; base < i1; base += kRowWarps) {
    // indices a batch ahead: the track of the next entity, the entity and point after it
    const uint32_t inext = base + kRowWarps + w, iafter = base + 2 * kRowWarps + w;
    uint32_t xa = 0, xl = 0, ye = 0, yp = 0;
    if (inext < i1) {
      xa = rt.pt_off[xp];
      xl = rt.pt_off[xp + 1] - xa;
    }
    if (iafter < i1) {
      ye = rt.ent[iafter];
      yp = rt.ent_point[iafter];
    }
    const uint32_t o = ce >> 1, ke = o - ca;
    const int cX = cl ? rt.seg_col[ce] : 0;
    for (uint32_t k0 = 0; __syncthreads_or(k0 < cl); k0 += kRowStage) {
      // ---- this warp's chunk: E (first round), targets, W ----
      // Loads are issued in two rounds: first every index (record offsets, target blocks and
      // columns, the point inverse), then every record value, so a chunk costs two memory latencies.
      const uint32_t Lc = k0 < cl ? min((uint32_t)kRowStage, cl - k0) : 0;
      const bool first = Lc && k0 == 0;
      const uint32_t rec_k = lane < Lc ? lin.obs_rec[ca + k0 + lane] : 0;  // record of chunk observation lane
      const uint32_t rec_o = first ? lin.obs_rec[o] : 0;
      int Y = -1, tcol = 0;
      uint32_t eid = 0;
      if (lane < 2 * Lc) {
        eid = 2 * (ca + k0 + (lane >> 1)) + (lane & 1);
        Y = rt.ent_block[eid];
        tcol = rt.seg_col[eid];
      }
      const double vi = (first && lane < 6) ? lin.vinv[6 * (size_t)cp + lane] : 0.0;
      // the entity's own record (E and the U term)
      double own = 0.0;
      if (first && lane < kRec) own = (double)lin.rec[rec_o + (size_t)lane * rs];
      // W of the chunk: lane kk + 16 h holds observation kk, columns 5h .. 5h + 4 (h = 1: 5 .. 8)
      const uint32_t kk = lane & 15, h = lane >> 4;
      const uint32_t rk_off = __shfl_sync(0xffffffffu, rec_k, (int)kk);
      const int c0 = h ? 5 : 0, nc = h ? 4 : 5;
      double jp[6], a0[5], a1[5];
      if (kk < Lc) {
        const R* rk = lin.rec + rk_off;
#pragma unroll
        for (int c = 0; c < 6; ++c) jp[c] = (double)rk[(size_t)(kJp + c) * rs];
#pragma unroll
        for (int j = 0; j < 5; ++j) {
          a0[j] = j < nc ? (double)rk[(size_t)(c0 + j) * rs] : 0.0;
          a1[j] = j < nc ? (double)rk[(size_t)(9 + c0 + j) * rs] : 0.0;
        }
      }
      if (first) {
        if (lane < kRec) Osh[w][lane] = own;
        if (lane < 6) Osh[w][kRec + lane] = vi;
      }
      if (kk < Lc) {
#pragma unroll
        for (int j = 0; j < 5; ++j)
          if (j < nc) {
            double* wq = Wsh[w][kk] + 3 * (c0 + j);
#pragma unroll
            for (int c = 0; c < 3; ++c) wq[c] = a0[j] * jp[c] + a1[j] * jp[3 + c];
          }
      }
      if (lane < 2 * Lc) {
        int sl = -1;
        uint32_t inf = 0;
        if (Y >= 0) {
          sl = nbr_local ? find_slot(nbr_s, 0, nn, Y) : find_slot(rt.nbr, n0, n1, Y);
          if (sl >= 0)
            inf = nbr_local ? ninf_s[sl]
                            : (uint32_t)(rt.slot_off[n0 + sl] - r0) << 3 | (uint32_t)rt.blk_dim[Y];
        }
        tsl[w][lane] = sl;
        tinf[w][lane] = inf;
        tcd[w][lane] = tcol | (k0 + (lane >> 1) == ke ? 1 << 8 : 0) | (int)(lane >> 1) << 9;
      }
      __syncwarp();
      if (first && lane < 3 * dX) {
        const int m = lane / 3, c = lane - 3 * m;
        const double* A = Osh[w];
        const double* P = Osh[w] + kRec;
        double wm[3];
        for (int d = 0; d < 3; ++d) wm[d] = A[cX + m] * A[kJp + d] + A[9 + cX + m] * A[kJp + 3 + d];
        const double v0 = c == 0 ? P[0] : (c == 1 ? P[1] : P[3]);
        const double v1 = c == 0 ? P[1] : (c == 1 ? P[2] : P[4]);
        const double v2 = c == 0 ? P[3] : (c == 1 ? P[4] : P[5]);
        Esh[w][lane] = wm[0] * v0 + wm[1] * v1 + wm[2] * v2;
      }
      if (lane == 0) {
        item_n[w] = 2 * (int)Lc;
        item_cx[w] = cX;
      }
      __syncthreads();
      // ---- every warp adds the batch's contributions to the slots it owns ----
      // One target is one FP64 m8n8k4 product on the tensor pipe, C (the slot, 8 x 8 with rows >= dX
      // and columns >= dY masked) += (-E) W_k,Y^T, plus A_o,X^T A_o,Y for the entity's own
      // observation. Fragments: lane l holds A(l / 4, l % 4), B(l % 4, l / 4) and C(l / 4, 2 (l % 4)
      // + i), i = 0, 1.
      const int fg = lane >> 2, ft = lane & 3;
      for (int b = 0; b < kRowWarps; ++b) {
        const int nt = item_n[b];
        if (nt == 0) continue;
        const int sl = lane < nt ? tsl[b][lane] : -1;
        unsigned mask = __ballot_sync(0xffffffffu, sl >= 0 && sl % kRowWarps == w);
        if (mask == 0u) continue;
        const int cxb = item_cx[b];
        const double* A = Osh[b];
        const double aE = (fg < dX && ft < 3) ? -Esh[b][3 * fg + ft] : 0.0;  // -E (dX x 3)
        const double aU = (fg < dX && ft < 2) ? A[9 * ft + cxb + fg] : 0.0;  // A_o,X^T (dX x 2)
        while (mask) {
          const int t = __ffs(mask) - 1;
          mask &= mask - 1;
          const uint32_t inf = tinf[b][t];
          const int cd = tcd[b][t], cY = cd & 0xff, own = (cd >> 8) & 1, dY = (int)(inf & 7);
          const double* Wk = Wsh[b][cd >> 9];
          double* out = row + (inf >> 3) + fg * dY;
          const double bW = (fg < dY && ft < 3) ? Wk[3 * (cY + fg) + ft] : 0.0;  // W_k,Y^T (3 x dY)
          const bool in0 = fg < dX && 2 * ft < dY, in1 = fg < dX && 2 * ft + 1 < dY;
          double c0 = in0 ? out[2 * ft] : 0.0, c1 = in1 ? out[2 * ft + 1] : 0.0;
          dmma_m8n8k4(aE, bW, c0, c1);
          if (own) {  // the same target in every lane
            const double bU = (fg < dY && ft < 2) ? A[9 * ft + cY + fg] : 0.0;  // A_o,Y (2 x dY)
            dmma_m8n8k4(aU, bU, c0, c1);
          }
          if (in0) out[2 * ft] = c0;
          if (in1) out[2 * ft + 1] = c1;
        }
      }
    }
    ce = xe;
    cp = xp;
    ca = xa;
    cl = inext < i1 ? xl : 0;
    xe = ye;
    xp = yp;
  }
  __syncthreads();
  if (row == row_sh)
    for (uint32_t k = tid; k < rlen; k += kRowThreads) rows[r0 + k] = row_sh[k];
}

// y = (S + lambda diag) x from the block rows: one warp per block row, lanes over the row's entries
// in a fixed assignment, then a fixed shuffle tree. With scale non-null the operator is the Jacobi-
// equilibrated D S D (D = diag(scale)) and lambda must be 0. With xy non-null, xy[CTA] = sum of
// x_b . y_b over the CTA's blocks in block order.
__global__ void __launch_bounds__(256) k_rows_matvec(RowTables rt, const double* __restrict__ rows,
                                                     const double* __restrict__ diag, double lambda,
                                                     const double* __restrict__ scale,
                                                     const double* __restrict__ x, double* __restrict__ y,
                                                     double* __restrict__ xy, const PcgCtl* ctl) {
  __shared__ double s_dot[8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int X = blockIdx.x * 8 + warp;
  const bool have = X < rt.nblocks;
  pdl_trigger();
  pdl_wait();
  if (pcg_stopped(ctl)) return;
  double dot = 0.0;
  if (have) {
    const int dX = rt.blk_dim[X], oX = rt.blk_off[X];
    const uint32_t n0 = rt.nbr_begin[X], n1 = rt.nbr_begin[X + 1];
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t q = n0 + lane; q < n1; q += 32) {
      const int Y = rt.nbr[q];
      const int dY = rt.blk_dim[Y], oY = rt.blk_off[Y];
      const double* S = rows + rt.slot_off[q];
      double xv[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) xv[c] = c < dY ? x[oY + c] * (scale ? scale[oY + c] : 1.0) : 0.0;
#pragma unroll
      for (int m = 0; m < 6; ++m)
        if (m < dX) {
          double s = 0.0;
#pragma unroll
          for (int c = 0; c < 6; ++c)
            if (c < dY) s += S[m * dY + c] * xv[c];
          acc[m] += s;
        }
    }
#pragma unroll
    for (int m = 0; m < 6; ++m) acc[m] = warp_sum(acc[m]);
    if (lane == 0) {
      for (int m = 0; m < dX; ++m) {
        double v = acc[m];
        if (scale) v *= scale[oX + m];
        v += lambda * diag[oX + m] * x[oX + m];
        y[oX + m] = v;
        dot += x[oX + m] * v;
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

// Diagonal of S (no damping) from the rows: thread per block, its own slot.
__global__ void k_rows_diag(RowTables rt, const double* __restrict__ rows, double* __restrict__ out) {
  const int X = blockIdx.x * blockDim.x + threadIdx.x;
  if (X >= rt.nblocks) return;
  const int dX = rt.blk_dim[X], oX = rt.blk_off[X];
  const int s = find_slot(rt.nbr, rt.nbr_begin[X], rt.nbr_begin[X + 1], X);
  const double* S = s >= 0 ? rows + rt.slot_off[rt.nbr_begin[X] + s] : nullptr;
  for (int m = 0; m < dX; ++m) out[oX + m] = S ? S[m * dX + m] : 0.0;
}

__global__ void k_set_int(int* p, int v) { *p = v; }

// ---- banded tiled matrix -----------------------------------------------------------------------
constexpr int kCT = 64;  // tile edge
constexpr int kCTT = kCT * kCT;

// Lower band of tiles of an n x n symmetric matrix in the permuted order: tile (i, j), 0 <= i - j <=
// bwt, at t + (i (bwt + 1) + (i - j)) kCTT, column-major inside the tile. Rows past n are padding
// (identity on the diagonal).
struct TileBand {
  int n, nt, bwt;
  double* t;
  double* w;  // nt tiles: the inverse of each diagonal tile of the factor (column-major)
};
__host__ __device__ __forceinline__ size_t tile_at(const TileBand& b, int i, int j) {
  return ((size_t)i * (b.bwt + 1) + (size_t)(i - j)) * kCTT;
}

// Scatter of the rows into the band: element (m, n) of block S_XY lands at permuted (P, Q) =
// (perm_off[X] + m, perm_off[Y] + n) when P >= Q. With scale non-null the stored value is
// scale_P S_PQ scale_Q; the diagonal gets + lambda diag_P, then - shift. One thread per entry.
__global__ void k_rows_to_tiles(RowTables rt, const double* __restrict__ rows, const int* __restrict__ perm_off,
                                const double* __restrict__ diag, double lambda, const double* __restrict__ scale,
                                double shift, TileBand tb) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= rt.entries) return;
  const int X = rt.nbr_row[q], Y = rt.nbr[q];
  const int dX = rt.blk_dim[X], dY = rt.blk_dim[Y];
  const int pX = perm_off[X], pY = perm_off[Y], oX = rt.blk_off[X], oY = rt.blk_off[Y];
  const double* S = rows + rt.slot_off[q];
  for (int m = 0; m < dX; ++m)
    for (int n = 0; n < dY; ++n) {
      const int P = pX + m, Q = pY + n;
      if (P < Q) continue;
      double v = S[m * dY + n];
      if (scale) v *= scale[oX + m] * scale[oY + n];
      if (P == Q) v += lambda * diag[oX + m] - shift;
      tb.t[tile_at(tb, P / kCT, Q / kCT) + (size_t)(Q % kCT) * kCT + (P % kCT)] = v;
    }
}

// Scatter of lower-triangle entries (row >= col) given as triplets into the band.
__global__ void k_triplets_to_tiles(uint32_t count, const int* __restrict__ rows, const int* __restrict__ cols,
                                    const double* __restrict__ vals, TileBand tb) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= count) return;
  const int P = rows[q], Q = cols[q];
  if (P < Q || P >= tb.n || Q < 0 || (P / kCT) - (Q / kCT) > tb.bwt) return;
  tb.t[tile_at(tb, P / kCT, Q / kCT) + (size_t)(Q % kCT) * kCT + (P % kCT)] = vals[q];
}

// Identity on the padding rows of the last diagonal tile.
__global__ void k_tiles_pad(TileBand tb) {
  const int r = tb.n + threadIdx.x;
  if (r >= tb.nt * kCT) return;
  const int i = tb.nt - 1;
  tb.t[tile_at(tb, i, i) + (size_t)(r % kCT) * kCT + (r % kCT)] = 1.0;
}

// Operands of the tile products are staged in shared memory with a padded row of kTS doubles (16-byte
// aligned rows; transposed stores hit 8 banks per warp instead of one).
constexpr int kTS = 66;
constexpr size_t kStagedTile = sizeof(double) * kCT * kTS;

// acc (4 x 4 per thread, 16 x 16 threads) += A B for 64 x 64 tiles staged as Ta[q * kTS + r] = A(r, q)
// and Tb[q * kTS + c] = B(q, c); the sum over q runs in order.
__device__ __forceinline__ void tile_mma_acc(const double* Ta, const double* Tb, double acc[4][4]) {
  const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
#pragma unroll 4
  for (int q = 0; q < kCT; ++q) {
    const double2 a01 = *reinterpret_cast<const double2*>(Ta + q * kTS + 4 * ty);
    const double2 a23 = *reinterpret_cast<const double2*>(Ta + q * kTS + 4 * ty + 2);
    const double2 b01 = *reinterpret_cast<const double2*>(Tb + q * kTS + 4 * tx);
    const double2 b23 = *reinterpret_cast<const double2*>(Tb + q * kTS + 4 * tx + 2);
    const double av[4] = {a01.x, a01.y, a23.x, a23.y}, bv[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] += av[a] * bv[b];
  }
}

// Stage the column-major tile g (element (r, c) at g[c * 64 + r]) as the operand M = g (flip false)
// or g^T (flip true), in the A layout (T[q * kTS + r] = M(r, q)) or the B layout (T[q * kTS + c] =
// M(q, c)). Global reads run along g's storage (coalesced).
__device__ __forceinline__ void stage_tile(const double* __restrict__ g, double* T, bool as_b, bool flip) {
  const bool direct = as_b == flip;  // A of g and B of g^T keep g's column-major order
  for (int w = threadIdx.x; w < kCTT; w += blockDim.x) {
    const int c = w / kCT, r = w - c * kCT;  // g(r, c)
    const double v = g[w];
    if (direct)
      T[c * kTS + r] = v;
    else
      T[r * kTS + c] = v;
  }
}

__device__ __forceinline__ void zero_acc(double acc[4][4]) {
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
}

// acc (output tile element (4 ty + a, 4 tx + b)) into a staged A operand: T[c * kTS + r] = scale acc(r, c)
__device__ __forceinline__ void acc_to_a(const double acc[4][4], double scale, double* T) {
  const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) T[(4 * tx + b) * kTS + 4 * ty + a] = scale * acc[a][b];
}

__device__ __forceinline__ void acc_store(const double acc[4][4], double* g) {
  const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
#pragma unroll
  for (int b = 0; b < 4; ++b)
#pragma unroll
    for (int a = 0; a < 4; ++a) g[(size_t)(4 * tx + b) * kCT + 4 * ty + a] = acc[a][b];
}

// POTRF of diagonal tile k and the inverse W_k = L_kk^-1 of its factor, both right-looking with the
// tile in registers: thread (ty, tx) of 16 x 16 holds elements (4 ty + a, 4 tx + b). Step j of the
// factorization publishes column j (its owners write it to shared memory, one barrier), and every
// thread scales it by 1 / sqrt(pivot) and updates its elements right of the column; step j of the
// inverse publishes the finished row j of W and every thread updates its rows below. The published
// buffers alternate, so each step takes one barrier. status[0] = 0 when a pivot is not finite and
// positive; later launches of the factorization then return at once.
__global__ void __launch_bounds__(256) k_tile_potrf(TileBand tb, int k, int* status) {
  __shared__ double Ls[kCT * (kCT + 1)];  // the tile in, then L (column-major, padded)
  __shared__ double pub[2][kCT];
  __shared__ double piv[2][3];  // pivot, its square root and the root's reciprocal
  __shared__ double rdiag[kCT];
  if (status[0] == 0) return;
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  double* g = tb.t + tile_at(tb, k, k);
  for (int w = tid; w < kCTT; w += blockDim.x) {
    const int c = w / kCT, r = w - c * kCT;
    Ls[c * (kCT + 1) + r] = g[w];
  }
  __syncthreads();
  double a[4][4];
#pragma unroll
  for (int ai = 0; ai < 4; ++ai)
#pragma unroll
    for (int bi = 0; bi < 4; ++bi) a[ai][bi] = Ls[(4 * tx + bi) * (kCT + 1) + 4 * ty + ai];
  for (int j = 0; j < kCT; ++j) {
    double* cj = pub[j & 1];
    if (tx == (j >> 2)) {  // static register indices: the column is picked by selects
      const int bj = j & 3;
#pragma unroll
      for (int ai = 0; ai < 4; ++ai) {
        const double v = bj == 0 ? a[ai][0] : (bj == 1 ? a[ai][1] : (bj == 2 ? a[ai][2] : a[ai][3]));
        cj[4 * ty + ai] = v;
        if (4 * ty + ai == j) {  // the diagonal's owner takes the root once for every thread
          const double r = sqrt(v);
          piv[j & 1][0] = v;
          piv[j & 1][1] = r;
          piv[j & 1][2] = 1.0 / r;
        }
      }
    }
    __syncthreads();
    const double d = piv[j & 1][0];  // the same value in every thread: all leave together
    if (!(isfinite(d) && d > 0.0)) {
      if (tid == 0) status[0] = 0;
      return;
    }
    const double sd = piv[j & 1][1], rs = piv[j & 1][2];
    // branch-free update: the multipliers of columns at or left of j are zero, so those columns keep
    // their values; elements above the diagonal take values that are never read (zeroed on output)
    double li[4], lc[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      li[q] = cj[4 * ty + q] * rs;
      lc[q] = 4 * tx + q > j ? cj[4 * tx + q] * rs : 0.0;
    }
#pragma unroll
    for (int ai = 0; ai < 4; ++ai)
#pragma unroll
      for (int bi = 0; bi < 4; ++bi) a[ai][bi] -= li[ai] * lc[bi];
    if (tx == (j >> 2)) {  // column j becomes the factor's column
#pragma unroll
      for (int bi = 0; bi < 4; ++bi)
        if (4 * tx + bi == j) {
#pragma unroll
          for (int ai = 0; ai < 4; ++ai) {
            const int i = 4 * ty + ai;
            if (i >= j) a[ai][bi] = i == j ? sd : li[ai];
          }
        }
    }
  }
  __syncthreads();  // every thread has read the last published column before Ls is rewritten
#pragma unroll
  for (int ai = 0; ai < 4; ++ai)
#pragma unroll
    for (int bi = 0; bi < 4; ++bi) {
      const int i = 4 * ty + ai, c = 4 * tx + bi;
      Ls[c * (kCT + 1) + i] = i >= c ? a[ai][bi] : 0.0;
    }
  __syncthreads();
  for (int w = tid; w < kCTT; w += blockDim.x) {
    const int c = w / kCT, r = w - c * kCT;
    g[w] = Ls[c * (kCT + 1) + r];
  }
  if (tid < kCT) rdiag[tid] = 1.0 / Ls[tid * (kCT + 1) + tid];
  // W = L^-1: row j of W is final once rows above it have been eliminated; it is published and the
  // rows below subtract L(i, j) times it
#pragma unroll
  for (int ai = 0; ai < 4; ++ai)
#pragma unroll
    for (int bi = 0; bi < 4; ++bi) a[ai][bi] = (4 * ty + ai == 4 * tx + bi) ? 1.0 : 0.0;
  __syncthreads();
  for (int j = 0; j < kCT; ++j) {
    double* xj = pub[j & 1];
    if (ty == (j >> 2)) {
      const int aj = j & 3;
      const double rd = rdiag[j];
#pragma unroll
      for (int ai = 0; ai < 4; ++ai)
        if (ai == aj) {
#pragma unroll
          for (int bi = 0; bi < 4; ++bi) {
            const double v = 4 * tx + bi <= j ? a[ai][bi] * rd : 0.0;
            a[ai][bi] = v;
            xj[4 * tx + bi] = v;
          }
        }
    }
    __syncthreads();
    // branch-free: the published row is zero right of column j and the multipliers are zero at or
    // above row j, so only the rows below j change, in the columns up to j
#pragma unroll
    for (int ai = 0; ai < 4; ++ai) {
      const int i = 4 * ty + ai;
      const double lij = i > j ? Ls[j * (kCT + 1) + i] : 0.0;
#pragma unroll
      for (int bi = 0; bi < 4; ++bi) a[ai][bi] -= lij * xj[4 * tx + bi];
    }
  }
  __syncthreads();  // Ls is reused to stage W for coalesced stores
#pragma unroll
  for (int ai = 0; ai < 4; ++ai)
#pragma unroll
    for (int bi = 0; bi < 4; ++bi) {
      const int i = 4 * ty + ai, c = 4 * tx + bi;
      Ls[c * (kCT + 1) + i] = i >= c ? a[ai][bi] : 0.0;
    }
  __syncthreads();
  double* wk = tb.w + (size_t)k * kCTT;
  for (int w = tid; w < kCTT; w += blockDim.x) {
    const int c = w / kCT, r = w - c * kCT;
    wk[w] = Ls[c * (kCT + 1) + r];
  }
}

// TRSM as a product: the tiles below diagonal tile k, L_ik = A_ik W_k^T (CTA per tile). Dynamic shared
// memory: two staged operands.
constexpr size_t kTrsmSmem = 2 * kStagedTile;
__global__ void __launch_bounds__(256) k_tile_trsm(TileBand tb, int k, const int* status) {
  extern __shared__ double shm[];
  if (status[0] == 0) return;
  double* Ta = shm;
  double* Tb = shm + kCT * kTS;
  const int i = k + 1 + blockIdx.x;
  double* bi = tb.t + tile_at(tb, i, k);
  stage_tile(bi, Ta, false, false);                       // A_ik
  stage_tile(tb.w + (size_t)k * kCTT, Tb, true, true);    // W_k^T
  __syncthreads();
  double acc[4][4];
  zero_acc(acc);
  tile_mma_acc(Ta, Tb, acc);
  acc_store(acc, bi);
}

// Trailing update of step k: A_ij -= L_ik L_jk^T for k < j <= i <= min(k + bwt, nt - 1), one CTA per
// tile, 16 x 16 threads with 4 x 4 outputs each; the sum over the tile's 64 columns runs in order.
constexpr size_t kUpdateSmem = 2 * kStagedTile;
__global__ void __launch_bounds__(256) k_tile_update(TileBand tb, int k, const int* status) {
  extern __shared__ double sh[];
  if (status[0] == 0) return;
  double* Ta = sh;
  double* Tb = sh + kCT * kTS;
  int idx = blockIdx.x;
  int ii = 0;
  while ((ii + 1) * (ii + 2) / 2 <= idx) ++ii;
  const int jj = idx - ii * (ii + 1) / 2;
  const int i = k + 1 + ii, j = k + 1 + jj;
  stage_tile(tb.t + tile_at(tb, i, k), Ta, false, false);  // L_ik
  stage_tile(tb.t + tile_at(tb, j, k), Tb, true, true);    // L_jk^T
  __syncthreads();
  double acc[4][4];
  zero_acc(acc);
  tile_mma_acc(Ta, Tb, acc);
  const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
  double* cij = tb.t + tile_at(tb, i, j);
#pragma unroll
  for (int b = 0; b < 4; ++b)
#pragma unroll
    for (int a = 0; a < 4; ++a) cij[(size_t)(4 * tx + b) * kCT + 4 * ty + a] -= acc[a][b];
}

// Forward (L y = b) and backward (L^T x = y) substitution with the banded tiled factor, one CTA of
// 256 threads, in place on the permuted vector v (n entries; the padding is not touched). Four
// threads per row of a tile sum the band's products in quarters, combined in a fixed order; the
// triangle inside a tile is solved by one warp with a fixed shuffle tree per row.
__device__ void tile_forward_rows(const TileBand& tb, double* v, int i, int j_lo, double* part, double* yt) {
  const int tid = threadIdx.x, r = tid & (kCT - 1), qtr = tid >> 6;  // 256 threads: 4 quarters
  double s = 0.0;
  const int j_first = max(j_lo, i - tb.bwt);
  for (int j = j_first; j < i; ++j) {
    const double* L = tb.t + tile_at(tb, i, j);
    for (int c = qtr; c < kCT; c += 4) s += L[(size_t)c * kCT + r] * v[j * kCT + c];
  }
  part[qtr * kCT + r] = s;
  __syncthreads();
  if (tid < kCT) {
    const int rr = tid;
    const int P = i * kCT + rr;
    const double b = P < tb.n ? v[P] : 0.0;
    yt[rr] = b - (((part[rr] + part[kCT + rr]) + part[2 * kCT + rr]) + part[3 * kCT + rr]);
  }
  __syncthreads();
  if (tid < 32) {  // in-tile forward solve, one warp
    const double* L = tb.t + tile_at(tb, i, i);
    for (int rr = 0; rr < kCT; ++rr) {
      double d = 0.0;
      for (int c = tid; c < rr; c += 32) d += L[(size_t)c * kCT + rr] * yt[c];
      d = warp_sum(d);
      if (tid == 0) yt[rr] = (yt[rr] - d) / L[(size_t)rr * kCT + rr];
      __syncwarp();
    }
  }
  __syncthreads();
  if (tid < kCT) {
    const int P = i * kCT + tid;
    if (P < tb.n) v[P] = yt[tid];
  }
  __syncthreads();
}

__global__ void __launch_bounds__(256) k_tile_solve(TileBand tb, double* v, const int* status) {
  __shared__ double part[4 * kCT];
  __shared__ double yt[kCT];
  if (status[0] == 0) return;
  const int tid = threadIdx.x, r = tid & (kCT - 1), qtr = tid >> 6;
  for (int i = 0; i < tb.nt; ++i) tile_forward_rows(tb, v, i, 0, part, yt);
  for (int i = tb.nt - 1; i >= 0; --i) {
    // x_i = L_ii^-T (y_i - sum_{j > i} L_ji^T x_j)
    double s = 0.0;
    const int j_last = min(tb.nt - 1, i + tb.bwt);
    for (int j = i + 1; j <= j_last; ++j) {
      const double* L = tb.t + tile_at(tb, j, i);
      for (int c = qtr; c < kCT; c += 4) {
        const int Q = j * kCT + c;
        if (Q < tb.n) s += L[(size_t)r * kCT + c] * v[Q];
      }
    }
    part[qtr * kCT + r] = s;
    __syncthreads();
    if (tid < kCT) {
      const int P = i * kCT + tid;
      const double b = P < tb.n ? v[P] : 0.0;
      yt[tid] = b - (((part[tid] + part[kCT + tid]) + part[2 * kCT + tid]) + part[3 * kCT + tid]);
    }
    __syncthreads();
    if (tid < 32) {  // in-tile backward solve with L_ii^T
      const double* L = tb.t + tile_at(tb, i, i);
      for (int rr = kCT - 1; rr >= 0; --rr) {
        double d = 0.0;
        for (int c = rr + 1 + tid; c < kCT; c += 32) d += L[(size_t)rr * kCT + c] * yt[c];
        d = warp_sum(d);
        if (tid == 0) yt[rr] = (yt[rr] - d) / L[(size_t)rr * kCT + rr];
        __syncwarp();
      }
    }
    __syncthreads();
    if (tid < kCT) {
      const int P = i * kCT + tid;
      if (P < tb.n) v[P] = yt[tid];
    }
    __syncthreads();
  }
}

// Gather / scatter between the original and the permuted parameter order.
__global__ void k_perm_gather(int n, const int* __restrict__ perm_to_orig, const double* __restrict__ src,
                              double sign, double* __restrict__ dst) {
  const int P = blockIdx.x * blockDim.x + threadIdx.x;
  if (P < n) dst[P] = sign * src[perm_to_orig[P]];
}
__global__ void k_perm_scatter(int n, const int* __restrict__ perm_to_orig, const double* __restrict__ src,
                               double* __restrict__ dst) {
  const int P = blockIdx.x * blockDim.x + threadIdx.x;
  if (P < n) dst[perm_to_orig[P]] = src[P];
}

// ---- selected inverse within the band (intrinsic marginal covariances) -----------------------
// Z = S^-1 restricted to the band of the factor, by the Takahashi recurrence on tiles, from the last
// tile column to the first: with Z L = L^-T,
//   Z_ij = -(sum_{k=j+1}^{j+bwt} Z_ik L_kj) L_jj^-1                      (i > j)
//   Z_jj = (L_jj^-T - sum_{k=j+1}^{j+bwt} Z_kj^T L_kj) L_jj^-1
// where Z_ik for i < k is Z_ki^T; every Z_ik needed lies in the band. The marginal covariance of a
// group is the block of Z at its parameters' positions (sparse/covariance.rs:564-587 gets the same
// block by solving S x = e_p column by column).
//
// Column j runs as three launches, so that the column's 64 x 64 products spread over the GPU:
//  k_takahashi_partial  CTA (b, s): part(b, s) = sum over k in chunk s of Z_ik L_kj, i = j + 1 + b,
//                       chunks of kTakahashiChunk consecutive k in order
//  k_takahashi_offdiag  CTA b: Z_ij = -(sum_s part(b, s)) W_j, and its share of the diagonal sum,
//                       q(b) = Z_ij^T L_ij
//  k_takahashi_diag     one CTA: Z_jj = (W_j^T - sum_b q(b)) W_j
// Every sum runs in a fixed order, so Z does not depend on scheduling. Dynamic shared memory:
// kTakahashiSmem (two staged operands).
constexpr size_t kTakahashiSmem = 2 * kStagedTile;
constexpr int kTakahashiChunk = 4;

// acc (output tile element (4 ty + a, 4 tx + b)) transposed into a staged A operand: A(c, r) = acc(r, c)
__device__ __forceinline__ void acc_to_at(const double acc[4][4], double* T) {
  const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) T[(4 * ty + a) * kTS + 4 * tx + b] = acc[a][b];
}

__global__ void __launch_bounds__(256) k_takahashi_partial(TileBand L, TileBand Z, int j, double* part,
                                                           const int* status) {
  extern __shared__ double sh[];
  if (status[0] == 0) return;
  double* Ta = sh;
  double* Tb = sh + kCT * kTS;
  const int i = j + 1 + blockIdx.x;
  const int kmax = min(L.nt - 1, j + L.bwt);
  const int k0 = j + 1 + kTakahashiChunk * blockIdx.y, k1 = min(kmax, k0 + kTakahashiChunk - 1);
  double acc[4][4];
  zero_acc(acc);
  for (int k = k0; k <= k1; ++k) {
    __syncthreads();
    if (i >= k)
      stage_tile(Z.t + tile_at(Z, i, k), Ta, false, false);  // Z_ik
    else
      stage_tile(Z.t + tile_at(Z, k, i), Ta, false, true);   // Z_ki^T
    stage_tile(L.t + tile_at(L, k, j), Tb, true, false);     // L_kj
    __syncthreads();
    tile_mma_acc(Ta, Tb, acc);
  }
  acc_store(acc, part + ((size_t)blockIdx.x * gridDim.y + blockIdx.y) * kCTT);
}

__global__ void __launch_bounds__(256) k_takahashi_offdiag(TileBand L, TileBand Z, int j, int nsplit,
                                                           const double* __restrict__ part, double* q,
                                                           const int* status) {
  extern __shared__ double sh[];
  if (status[0] == 0) return;
  double* Ta = sh;
  double* Tb = sh + kCT * kTS;
  const int i = j + 1 + blockIdx.x;
  // -(sum of the partial tiles, in order) into the A operand, read along the tiles' storage
  const double* pb = part + (size_t)blockIdx.x * nsplit * kCTT;
  for (int w = threadIdx.x; w < kCTT; w += blockDim.x) {
    double v = 0.0;
    for (int s = 0; s < nsplit; ++s) v += pb[(size_t)s * kCTT + w];
    Ta[(w / kCT) * kTS + (w % kCT)] = -v;
  }
  stage_tile(L.w + (size_t)j * kCTT, Tb, true, false);  // W_j
  __syncthreads();
  double acc[4][4];
  zero_acc(acc);
  tile_mma_acc(Ta, Tb, acc);
  acc_store(acc, Z.t + tile_at(Z, i, j));
  __syncthreads();
  acc_to_at(acc, Ta);                                    // Z_ij^T
  stage_tile(L.t + tile_at(L, i, j), Tb, true, false);  // L_ij
  __syncthreads();
  zero_acc(acc);
  tile_mma_acc(Ta, Tb, acc);
  acc_store(acc, q + (size_t)blockIdx.x * kCTT);
}

__global__ void __launch_bounds__(256) k_takahashi_diag(TileBand L, TileBand Z, int j, int m,
                                                        const double* __restrict__ q, const int* status) {
  extern __shared__ double sh[];
  if (status[0] == 0) return;
  double* Ta = sh;
  double* Tb = sh + kCT * kTS;
  // -(sum of the tiles' shares, in order) into the A operand, read along the tiles' storage
  for (int w = threadIdx.x; w < kCTT; w += blockDim.x) {
    double v = 0.0;
    for (int b = 0; b < m; ++b) v += q[(size_t)b * kCTT + w];
    Ta[(w / kCT) * kTS + (w % kCT)] = -v;
  }
  const double* wj = L.w + (size_t)j * kCTT;
  __syncthreads();
  for (int w = threadIdx.x; w < kCTT; w += blockDim.x) {  // + W_j^T: A(r, q) += W(q, r)
    const int c = w / kCT, r = w - c * kCT;                // W(r, c) at wj[w]
    Ta[r * kTS + c] += wj[w];                              // A element (c, r) of the operand
  }
  double acc[4][4];
  stage_tile(wj, Tb, true, false);  // W_j
  __syncthreads();
  zero_acc(acc);
  tile_mma_acc(Ta, Tb, acc);
  acc_store(acc, Z.t + tile_at(Z, j, j));
}

// (S^-1)_gg of each free group from Z: 9 values per group (row-major), thread per group.
__global__ void k_z_marginals(TileBand Z, int ngroups, const int* __restrict__ pos, const int* __restrict__ dims,
                              double* __restrict__ out, const int* status) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroups || status[0] == 0) return;
  const int dim = dims[g];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double v = 0.0;
      if (a < dim && b < dim) {
        int P = pos[3 * g + a], Q = pos[3 * g + b];
        if (P < Q) {
          const int t = P;
          P = Q;
          Q = t;
        }
        v = Z.t[tile_at(Z, P / kCT, Q / kCT) + (size_t)(Q % kCT) * kCT + (P % kCT)];
      }
      out[9 * (size_t)g + 3 * a + b] = v;
    }
}

// Largest |eigenvalue| of the equilibrated D S D by power iteration (Rayleigh quotient of the
// normalized iterate), one CTA of 1024 threads running every iteration, so the host waits once:
// out[0] = lambda, out[1] = 1 when it settled (|rq - lambda| <= 1e-10 |rq| after the 8th iteration) or
// ran its 200 iterations with finite values, 0 otherwise. v, w: n doubles of scratch.
__global__ void __launch_bounds__(1024) k_power_iteration(RowTables rt, const double* __restrict__ rows,
                                                          const double* __restrict__ scale, int n, double* v,
                                                          double* w, double* out) {
  __shared__ double red[32][2];
  __shared__ double s_nrm, s_rq;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double v0 = 1.0 / sqrt((double)n);
  for (int i = tid; i < n; i += blockDim.x) v[i] = v0;
  __syncthreads();
  double lam = 0.0;
  int ok = 0;
  for (int it = 0; it < 200; ++it) {
    // w = D S D v: warp per block row
    for (int X = warp; X < rt.nblocks; X += 32) {
      const int dX = rt.blk_dim[X], oX = rt.blk_off[X];
      const uint32_t n0 = rt.nbr_begin[X], n1 = rt.nbr_begin[X + 1];
      double acc[6] = {0, 0, 0, 0, 0, 0};
      for (uint32_t q = n0 + lane; q < n1; q += 32) {
        const int Y = rt.nbr[q];
        const int dY = rt.blk_dim[Y], oY = rt.blk_off[Y];
        const double* S = rows + rt.slot_off[q];
        for (int m = 0; m < dX; ++m) {
          double s = 0.0;
          for (int c = 0; c < dY; ++c) s += S[m * dY + c] * (scale[oY + c] * v[oY + c]);
          acc[m] += s;
        }
      }
      for (int m = 0; m < 6; ++m) acc[m] = warp_sum(acc[m]);
      if (lane == 0)
        for (int m = 0; m < dX; ++m) w[oX + m] = acc[m] * scale[oX + m];
    }
    __syncthreads();
    double nn = 0.0, rq = 0.0;
    for (int i = tid; i < n; i += blockDim.x) {
      nn += w[i] * w[i];
      rq += v[i] * w[i];
    }
    nn = warp_sum(nn);
    rq = warp_sum(rq);
    if (lane == 0) {
      red[warp][0] = nn;
      red[warp][1] = rq;
    }
    __syncthreads();
    if (tid == 0) {
      double a = 0.0, b = 0.0;
      for (int k = 0; k < 32; ++k) {
        a += red[k][0];
        b += red[k][1];
      }
      s_nrm = sqrt(a);
      s_rq = b;
    }
    __syncthreads();
    const double nrm = s_nrm, q = s_rq;
    if (!(isfinite(nrm) && nrm > 0.0)) {
      ok = 0;
      break;
    }
    const bool settled = it > 8 && fabs(q - lam) <= 1e-10 * fabs(q);
    lam = q;
    for (int i = tid; i < n; i += blockDim.x) v[i] = w[i] / nrm;
    __syncthreads();
    ok = 1;
    if (settled) break;
  }
  if (tid == 0) {
    out[0] = lam;
    out[1] = ok;
  }
}

}  // namespace omvgba
