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

constexpr int kRowThreads = 128;

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

// Row X of S. For each entity e of X (observation o at point p, camera columns cX..cX+dX) and each
// entity e' of p in block Y (observation o', columns cY..): S_XY += Jc_e^T M Jc_e' with the 2 x 2
// M = [o == o'] I - Jp_o Vhat_p^-1 Jp_o'^T (U, the pose/intrinsic edges and the point coupling in one
// term). Targets of one point that fall in the same block are summed in target order by one thread
// per element; entities are taken one after another, so every element is accumulated in entity
// order. FP64 accumulation from records of type R.
//
// Latency: a CTA walks thousands of entities one after another, so the per-entity chain is kept
// short: the records of a track of up to kRowStage observations are staged in shared memory (longer
// tracks are read from global memory), the block's neighbour list sits in shared memory when it has
// at most kRowNbr entries, and thread 0 fetches the next entity's indices while the current one is
// computed. Small static shared memory keeps many CTAs resident. Dynamic shared memory: 4 x
// max_track ints (the target slots and columns).
constexpr int kRowStage = 32;
constexpr int kRowNbr = 1024;
template <typename R>
__global__ void __launch_bounds__(kRowThreads) k_block_rows(RowTables rt, LinOut<R> lin, int max_track,
                                                            double* __restrict__ rows) {
  extern __shared__ int ish[];
  int* tslot = ish;                  // per target: slot or -1
  int* tcol = ish + 2 * max_track;   // per target: column of its segment
  __shared__ double jr[kRowStage * kRec];  // the point's records (tracks of at most kRowStage)
  __shared__ int nbr_s[kRowNbr];
  __shared__ double G[6];                  // Jp_o Vhat^-1 (2 x 3)
  __shared__ double aX[12];                // the entity's 2 x dX camera columns
  __shared__ uint32_t s_ent[2][4];         // current / next entity: e, point, first observation, track length
  const int X = blockIdx.x, tid = threadIdx.x;
  if (X >= rt.nblocks) return;
  const int dX = rt.blk_dim[X];
  const uint32_t n0 = rt.nbr_begin[X], n1 = rt.nbr_begin[X + 1];
  const bool nbr_local = n1 - n0 <= (uint32_t)kRowNbr;
  if (nbr_local)
    for (uint32_t k = tid; k < n1 - n0; k += blockDim.x) nbr_s[k] = rt.nbr[n0 + k];
  const uint64_t r0 = rt.slot_off[n0], r1 = rt.slot_off[n1];
  for (uint64_t k = r0 + tid; k < r1; k += blockDim.x) rows[k] = 0.0;
  const uint32_t i0 = rt.blk_ent[X], i1 = rt.blk_ent[X + 1];
  if (tid == 0 && i0 < i1) {
    const uint32_t e = rt.ent[i0], p = rt.ent_point[i0];
    const uint32_t a = rt.pt_off[p], b = rt.pt_off[p + 1];
    s_ent[0][0] = e;
    s_ent[0][1] = p;
    s_ent[0][2] = a;
    s_ent[0][3] = b - a;
  }
  const int rs = lin.rs;
  for (uint32_t i = i0; i < i1; ++i) {
    __syncthreads();  // the previous entity is finished (and the row is zeroed, the list staged)
    const int buf = (i - i0) & 1;
    const uint32_t e = s_ent[buf][0], o = e >> 1, p = s_ent[buf][1], o0 = s_ent[buf][2], L = s_ent[buf][3];
    const bool staged = L <= (uint32_t)kRowStage;
    if (staged)
      for (uint32_t k = tid; k < (uint32_t)kRec * L; k += blockDim.x) {
        const uint32_t c = k / L, j = k - c * L;
        jr[j * kRec + c] = (double)lin.rec[lin.obs_rec[o0 + j] + (size_t)c * rs];
      }
    for (uint32_t t = tid; t < 2 * L; t += blockDim.x) {
      const uint32_t eid = 2 * (o0 + (t >> 1)) + (t & 1);
      const int Y = rt.ent_block[eid];
      int sl = -1;
      if (Y >= 0) sl = nbr_local ? find_slot(nbr_s, 0, n1 - n0, Y) : find_slot(rt.nbr, n0, n1, Y);
      tslot[t] = sl;
      tcol[t] = rt.seg_col[eid];
    }
    if (tid == 32 && i + 1 < i1) {  // the next entity's indices, fetched while this one is computed
      const uint32_t en = rt.ent[i + 1], pn = rt.ent_point[i + 1];
      const uint32_t a = rt.pt_off[pn], b = rt.pt_off[pn + 1];
      s_ent[buf ^ 1][0] = en;
      s_ent[buf ^ 1][1] = pn;
      s_ent[buf ^ 1][2] = a;
      s_ent[buf ^ 1][3] = b - a;
    }
    const uint32_t jo = o - o0;
    if (tid == 0) {
      const double* vi = lin.vinv + 6 * (size_t)p;
      const double Vi[6] = {vi[0], vi[1], vi[2], vi[3], vi[4], vi[5]};
      const R* ro = lin.rec + lin.obs_rec[o];
      double jp[6];
      for (int k = 0; k < 6; ++k) jp[k] = (double)ro[(size_t)(kJp + k) * rs];
      sym3_apply(Vi, jp, G);
      sym3_apply(Vi, jp + 3, G + 3);
      const int cX = rt.seg_col[e];
      for (int m = 0; m < 6; ++m) {
        aX[m] = m < dX ? (double)ro[(size_t)(cX + m) * rs] : 0.0;
        aX[6 + m] = m < dX ? (double)ro[(size_t)(9 + cX + m) * rs] : 0.0;
      }
    }
    __syncthreads();
    for (uint32_t w = tid; w < 2 * L * 36; w += blockDim.x) {
      const uint32_t t = w / 36, mn = w - 36 * t, m = mn / 6, n = mn - 6 * m;
      const int sl = tslot[t];
      if (sl < 0 || (int)m >= dX) continue;
      const int dY = rt.blk_dim[nbr_local ? nbr_s[sl] : rt.nbr[n0 + sl]];
      if ((int)n >= dY) continue;
      bool leader = true;
      for (uint32_t t2 = 0; t2 < t; ++t2) leader = leader && tslot[t2] != sl;
      if (!leader) continue;
      const double a0 = aX[m], a1 = aX[6 + m];
      double acc = 0.0;
      for (uint32_t t2 = t; t2 < 2 * L; ++t2) {
        if (tslot[t2] != sl) continue;
        const uint32_t j = t2 >> 1;
        const int cY = tcol[t2];
        double q[6], b0, b1;
        if (staged) {
          const double* rj = jr + j * kRec;
          for (int k = 0; k < 6; ++k) q[k] = rj[kJp + k];
          b0 = rj[cY + n];
          b1 = rj[9 + cY + n];
        } else {
          const R* rj = lin.rec + lin.obs_rec[o0 + j];
          for (int k = 0; k < 6; ++k) q[k] = (double)rj[(size_t)(kJp + k) * rs];
          b0 = (double)rj[(size_t)(cY + n) * rs];
          b1 = (double)rj[(size_t)(9 + cY + n) * rs];
        }
        double M00 = -(G[0] * q[0] + G[1] * q[1] + G[2] * q[2]);
        double M01 = -(G[0] * q[3] + G[1] * q[4] + G[2] * q[5]);
        double M10 = -(G[3] * q[0] + G[4] * q[1] + G[5] * q[2]);
        double M11 = -(G[3] * q[3] + G[4] * q[4] + G[5] * q[5]);
        if (j == jo) {
          M00 += 1.0;
          M11 += 1.0;
        }
        acc += a0 * (M00 * b0 + M01 * b1) + a1 * (M10 * b0 + M11 * b1);
      }
      rows[rt.slot_off[n0 + sl] + m * dY + n] += acc;
    }
  }
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

// POTRF of diagonal tile k (right-looking inside the tile) and the inverse W_k = L_kk^-1 of its factor
// (column by column, forward substitution). status[0] = 0 when a pivot is not finite and positive;
// later launches of the factorization then return at once.
__global__ void __launch_bounds__(256) k_tile_potrf(TileBand tb, int k, int* status) {
  __shared__ double A[kCT * (kCT + 1)];
  __shared__ int fail;
  if (status[0] == 0) return;
  const int tid = threadIdx.x;
  double* g = tb.t + tile_at(tb, k, k);
  for (int w = tid; w < kCTT; w += blockDim.x) {
    const int c = w / kCT, r = w - c * kCT;
    A[c * (kCT + 1) + r] = g[w];
  }
  if (tid == 0) fail = 0;
  for (int j = 0; j < kCT; ++j) {
    __syncthreads();
    if (tid == 0) {
      const double d = A[j * (kCT + 1) + j];
      if (!(isfinite(d) && d > 0.0))
        fail = 1;
      else
        A[j * (kCT + 1) + j] = sqrt(d);
    }
    __syncthreads();
    if (fail) break;
    const double piv = A[j * (kCT + 1) + j];
    for (int i = j + 1 + tid; i < kCT; i += blockDim.x) A[j * (kCT + 1) + i] /= piv;
    __syncthreads();
    const int m = kCT - j - 1;
    for (int w = tid; w < m * m; w += blockDim.x) {
      const int c = j + 1 + w / m, i = j + 1 + w % m;
      if (c <= i) A[c * (kCT + 1) + i] -= A[j * (kCT + 1) + i] * A[j * (kCT + 1) + c];
    }
  }
  __syncthreads();
  if (fail) {
    if (tid == 0) status[0] = 0;
    return;
  }
  for (int w = tid; w < kCTT; w += blockDim.x) {
    const int c = w / kCT, r = w - c * kCT;
    g[w] = r >= c ? A[c * (kCT + 1) + r] : 0.0;
  }
  if (tid < kCT) {  // column c of W: L w = e_c, rows c..63
    const int c = tid;
    double* wc = tb.w + (size_t)k * kCTT + (size_t)c * kCT;
    for (int r = 0; r < c; ++r) wc[r] = 0.0;
    double x[kCT];
    for (int r = c; r < kCT; ++r) {
      double v = r == c ? 1.0 : 0.0;
      for (int m = c; m < r; ++m) v -= A[m * (kCT + 1) + r] * x[m];
      x[r] = v / A[r * (kCT + 1) + r];
      wc[r] = x[r];
    }
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
// Off-diagonal tiles of Z in column j: CTA per i in (j, min(j + bwt, nt - 1)]: acc = sum_k Z_ik L_kj,
// then Z_ij = -acc W_j. Dynamic shared memory: kTakahashiSmem (two staged operands).
constexpr size_t kTakahashiSmem = 2 * kStagedTile;
__global__ void __launch_bounds__(256) k_takahashi_offdiag(TileBand L, TileBand Z, int j, const int* status) {
  extern __shared__ double sh[];
  if (status[0] == 0) return;
  double* Ta = sh;
  double* Tb = sh + kCT * kTS;
  const int i = j + 1 + blockIdx.x;
  const int kmax = min(L.nt - 1, j + L.bwt);
  double acc[4][4];
  zero_acc(acc);
  for (int k = j + 1; k <= kmax; ++k) {
    __syncthreads();
    if (i >= k)
      stage_tile(Z.t + tile_at(Z, i, k), Ta, false, false);  // Z_ik
    else
      stage_tile(Z.t + tile_at(Z, k, i), Ta, false, true);   // Z_ki^T
    stage_tile(L.t + tile_at(L, k, j), Tb, true, false);     // L_kj
    __syncthreads();
    tile_mma_acc(Ta, Tb, acc);
  }
  __syncthreads();
  acc_to_a(acc, -1.0, Ta);
  stage_tile(L.w + (size_t)j * kCTT, Tb, true, false);  // W_j
  __syncthreads();
  zero_acc(acc);
  tile_mma_acc(Ta, Tb, acc);
  acc_store(acc, Z.t + tile_at(Z, i, j));
}

// Diagonal tile of Z in column j (after its off-diagonal tiles): acc = sum_k Z_kj^T L_kj, then
// Z_jj = (W_j^T - acc) W_j. One CTA.
__global__ void __launch_bounds__(256) k_takahashi_diag(TileBand L, TileBand Z, int j, const int* status) {
  extern __shared__ double sh[];
  if (status[0] == 0) return;
  double* Ta = sh;
  double* Tb = sh + kCT * kTS;
  const int kmax = min(L.nt - 1, j + L.bwt);
  double acc[4][4];
  zero_acc(acc);
  for (int k = j + 1; k <= kmax; ++k) {
    __syncthreads();
    stage_tile(Z.t + tile_at(Z, k, j), Ta, false, true);  // Z_kj^T
    stage_tile(L.t + tile_at(L, k, j), Tb, true, false);  // L_kj
    __syncthreads();
    tile_mma_acc(Ta, Tb, acc);
  }
  __syncthreads();
  acc_to_a(acc, -1.0, Ta);  // -acc
  const double* wj = L.w + (size_t)j * kCTT;
  __syncthreads();
  for (int w = threadIdx.x; w < kCTT; w += blockDim.x) {  // + W_j^T: A(r, q) += W(q, r)
    const int c = w / kCT, r = w - c * kCT;                // W(r, c) at wj[w]
    Ta[r * kTS + c] += wj[w];                              // A element (c, r) of the operand
  }
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
