// canon.cu -- canonicalize! and generate! on device tableaux.
//
// canonicalize! (src/canonicalization.jl:95-133) is Garcia's two-stage
// elimination: for every column j (X bits, then Z bits) find the first row at
// or below the current pivot position i with the bit set, swap it to i, and
// left-multiply every other row that has the bit by the pivot row.  The
// pivot steps are serial, so the kernel is one thread-block cluster that stays
// resident for the whole elimination:
//   - the rows are split over the cluster's CTAs and held in shared memory
//     (row stride W+1 words, so a thread-per-row column probe and a
//     warp-per-row update are both bank-conflict free); tableaux too tall for
//     the cluster's shared memory stay in global memory (L2) instead;
//   - rows never move: a row swap only exchanges logical positions (pos[] per
//     CTA, inv[] replicated in every CTA), and rows are written to their final
//     positions at the end;
//   - per column each CTA reduces its local candidate (smallest position >= i
//     with the bit) with __reduce_min_sync, publishes it in shared memory, and
//     after one cluster barrier every CTA reads all candidates through
//     distributed shared memory; the pivot row is fetched the same way.
// The row products keep the reference's phase arithmetic exactly
// (mul_left!(state, m, i): phase_m <- (s + phase_m + phase_i) mod 4).
#include <cooperative_groups.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "qcb_internal.h"

namespace cg = cooperative_groups;

namespace qcb {

__device__ __forceinline__ void mul_step_c(uint64_t x1, uint64_t z1, uint64_t& x2, uint64_t& z2,
                                           uint64_t& c1, uint64_t& c2) {
  const uint64_t nx = x1 ^ x2, nz = z1 ^ z2;
  const uint64_t x1z2 = x1 & z2;
  const uint64_t anti = (x2 & z1) ^ x1z2;
  c2 ^= (c1 ^ nx ^ nz ^ x1z2) & anti;
  c1 ^= anti;
  x2 = nx;
  z2 = nz;
}

// Elimination modes of canon_kernel.
enum : uint32_t {
  ELIM_BOTH = 0,  // canonicalize!: X stage then Z stage over all columns
  ELIM_X = 1,     // canonicalize_gott! first stage: X stage only
  ELIM_Z = 2,     // canonicalize_gott! second stage: Z stage from column c0, pivots from row i0
  ELIM_RREF = 3   // canonicalize_rref!: X then Z per listed column, pivots from the last row upwards
};

struct CanonArgs {
  uint64_t* xzs;   // first row of the stabilizer view
  uint8_t* ph;
  uint64_t* dxzs;  // destabilizer rows paired with the view rows (Destabilizer kinds), or null
  uint8_t* dph;
  uint32_t rows, n, W;
  uint32_t RB;     // rows per CTA
  int phases;
  int smem_rows;   // 1: rows staged in shared memory
  uint64_t* gtmp;  // global mode: permuted output (view rows, then destabilizer rows)
  uint8_t* gtmp_ph;
  int32_t* out;    // [0] pivots of the X stage (ELIM_BOTH) or of the launch, [1] next pivot position
  uint32_t mode, c0, i0;
  const uint32_t* cols;  // ELIM_RREF columns, 0-based
  uint32_t ncols;
  int32_t* pivcols;      // column of every pivot in order, or null
  int32_t copy_back;     // global mode in a batch: the body copies gtmp back into the tableau
  int32_t pad_;
};

constexpr uint32_t CANON_THREADS = 1024;

// D: destabilizer rows ride along; DESC: pivots from the last row upwards
// (canonicalize_rref!).  Compile-time so that canonicalize! runs the lean
// instance.
template <bool D, bool DESC>
__device__ __forceinline__ void canon_body(const CanonArgs& a, uint64_t* smem) {
  cg::cluster_group cl = cg::this_cluster();
  const uint32_t me = cl.block_rank();
  const uint32_t CS = cl.num_blocks();
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const uint32_t W = a.W, len = W / 2, WS = W + 1;
  const uint32_t r0 = me * a.RB;
  const uint32_t nloc = r0 < a.rows ? min(a.RB, a.rows - r0) : 0u;

  uint64_t* piv = smem;                                               // W words
  uint64_t* rowsbuf = piv + W + 1;                                    // RB * WS words (smem mode)
  uint64_t* drows = rowsbuf + (a.smem_rows ? (size_t)a.RB * WS : 0);  // RB * WS words (smem mode, D)
  uint64_t* part = drows + (a.smem_rows && D ? (size_t)a.RB * WS : 0);  // 2 x W words (D)
  uint32_t* slot = (uint32_t*)(part + (D ? 2 * (size_t)W : 0));       // 2 candidate slots
  uint32_t* red = slot + 2;                                           // 32 warp minima
  uint32_t* ctl = red + 32;                                           // [0]=k [1]=pstar [2]=piv phase
  uint32_t* inv = ctl + 4;                                            // rows (replicated)
  uint32_t* pos = inv + a.rows;                                       // RB
  uint8_t* lph = (uint8_t*)(pos + a.RB);                              // RB
  uint8_t* dlph = lph + a.RB;                                         // RB (D)

  auto ROW = [&](uint32_t r) -> uint64_t* {
    return a.smem_rows ? rowsbuf + (size_t)r * WS : a.xzs + (size_t)(r0 + r) * W;
  };
  auto DROW = [&](uint32_t r) -> uint64_t* {
    return a.smem_rows ? drows + (size_t)r * WS : a.dxzs + (size_t)(r0 + r) * W;
  };

  for (uint32_t r = tid; r < nloc; r += blockDim.x) {
    pos[r] = r0 + r;
    lph[r] = a.ph[r0 + r];
    if (D) dlph[r] = a.dph[r0 + r];
  }
  if (a.smem_rows) {
    for (uint32_t r = warp; r < nloc; r += nwarps)
      for (uint32_t w = lane; w < W; w += 32) {
        rowsbuf[(size_t)r * WS + w] = a.xzs[(size_t)(r0 + r) * W + w];
        if (D) drows[(size_t)r * WS + w] = a.dxzs[(size_t)(r0 + r) * W + w];
      }
  }
  for (uint32_t p = tid; p < a.rows; p += blockDim.x) inv[p] = p;
  cl.sync();

  // The destabilizer update of mul_left!(state, m, i) (destabilizer i <- m * i,
  // no phase) XORs the destabilizer rows of every eliminated row into the
  // pivot's.  Each CTA accumulates its rows' share in part[parity]; the pivot
  // row's owner folds the cluster's shares in after the next cluster barrier
  // (before it can read that row again).
  bool pend = false;
  uint32_t pend_par = 0, pend_owner = 0, pend_lr = 0;
  auto fold_pending = [&]() {
    if (pend && me == pend_owner) {
      uint64_t* dst = DROW(pend_lr);
      for (uint32_t w = tid; w < W; w += blockDim.x) {
        uint64_t x = 0;
        for (uint32_t q = 0; q < CS; q++) x ^= *cl.map_shared_rank(part + (size_t)pend_par * W + w, q);
        dst[w] ^= x;
      }
    }
    pend = false;
  };

  constexpr bool desc = DESC;
  const uint32_t nsteps = desc ? 2 * a.ncols
                               : (a.mode == ELIM_BOTH ? 2 * a.n : (a.mode == ELIM_X ? a.n : (a.n > a.c0 ? a.n - a.c0 : 0u)));
  int32_t i = desc ? (int32_t)a.rows - 1 : (int32_t)a.i0;  // next pivot position
  uint32_t rx = 0, step = 0, npiv = 0;
  for (uint32_t t = 0; t < nsteps; t++) {
    uint32_t stage, j;
    if (desc) {
      j = a.cols[t >> 1];
      stage = t & 1;
    } else if (a.mode == ELIM_BOTH) {
      stage = t >= a.n;
      j = stage ? t - a.n : t;
      if (t == a.n) rx = (uint32_t)i;
    } else if (a.mode == ELIM_X) {
      stage = 0;
      j = t;
    } else {
      stage = 1;
      j = a.c0 + t;
    }
    // the search range [i, rows) (or [0, i] from the bottom) is empty
    if (desc ? i < 0 : i >= (int32_t)a.rows) continue;
    const uint32_t lo = desc ? 0u : (uint32_t)i, hi = desc ? (uint32_t)i : a.rows - 1;
    const uint32_t wj = stage * len + (j >> 6);
    const uint64_t bm = 1ull << (j & 63);
    // local candidate: smallest position in [lo, hi] with the bit set
    uint32_t best = 0xFFFFFFFFu;
    for (uint32_t r = tid; r < nloc; r += blockDim.x) {
      const uint32_t p = pos[r];
      const bool in = desc ? p <= hi : p >= lo;  // the other end of the range is the tableau's
      if (in && (ROW(r)[wj] & bm)) best = min(best, p);
    }
    best = __reduce_min_sync(0xFFFFFFFFu, best);
    if (lane == 0) red[warp] = best;
    __syncthreads();
    if (warp == 0) {
      uint32_t b = lane < nwarps ? red[lane] : 0xFFFFFFFFu;
      b = __reduce_min_sync(0xFFFFFFFFu, b);
      if (lane == 0) slot[step & 1] = b;
    }
    cl.sync();
    fold_pending();
    if (warp == 0) {
      // the cluster's candidates, one CTA per lane
      uint32_t k = lane < CS ? *cl.map_shared_rank(&slot[step & 1], lane) : 0xFFFFFFFFu;
      k = __reduce_min_sync(0xFFFFFFFFu, k);
      if (lane == 0) ctl[0] = k;
      if (lane == 0 && k != 0xFFFFFFFFu) {
        // rowswap!(state, k, i) on logical positions
        const uint32_t pstar = inv[k], aphys = inv[i];
        inv[i] = pstar;
        inv[k] = aphys;
        if (pstar >= r0 && pstar < r0 + nloc) pos[pstar - r0] = (uint32_t)i;
        if (aphys >= r0 && aphys < r0 + nloc) pos[aphys - r0] = k;
        ctl[1] = pstar;
      }
    }
    __syncthreads();
    step++;
    const uint32_t k = ctl[0];
    if (k == 0xFFFFFFFFu) continue;
    const uint32_t pstar = ctl[1];
    const uint32_t owner = pstar / a.RB, lr = pstar - owner * a.RB;
    const uint32_t par = npiv & 1;
    {
      const uint64_t* src;
      const uint8_t* srcph;
      if (a.smem_rows) {
        uint64_t* base = rowsbuf + (size_t)lr * WS;
        uint8_t* pb = lph + lr;
        src = owner == me ? base : cl.map_shared_rank(base, owner);
        srcph = owner == me ? pb : cl.map_shared_rank(pb, owner);
      } else {
        src = a.xzs + (size_t)pstar * W;
        uint8_t* pb = lph + lr;
        srcph = owner == me ? pb : cl.map_shared_rank(pb, owner);
      }
      for (uint32_t w = tid; w < W; w += blockDim.x) {
        piv[w] = src[w];
        if (D) part[(size_t)par * W + w] = 0;
      }
      if (tid == 0) ctl[2] = *srcph;
    }
    __syncthreads();
    const uint32_t pph = ctl[2];
    for (uint32_t r = warp; r < nloc; r += nwarps) {
      if (r0 + r == pstar) continue;
      uint64_t* row = ROW(r);
      if (!(row[wj] & bm)) continue;
      uint64_t c1 = 0, c2 = 0;
      for (uint32_t w = lane; w < len; w += 32) {
        uint64_t x2 = row[w], z2 = row[len + w];
        mul_step_c(piv[w], piv[len + w], x2, z2, c1, c2);
        row[w] = x2;
        row[len + w] = z2;
      }
      if (a.phases) {
        const uint32_t s =
            __reduce_add_sync(0xFFFFFFFFu, (uint32_t)(__popcll(c1) + 2 * __popcll(c2)) & 3u) & 3u;
        if (lane == 0) lph[r] = (uint8_t)((s + lph[r] + pph) & 3u);
      }
      if (D) {
        const uint64_t* dr = DROW(r);
        for (uint32_t w = lane; w < W; w += 32)
          atomicXor((unsigned long long*)(part + (size_t)par * W + w), (unsigned long long)dr[w]);
      }
    }
    __syncthreads();
    if (D) {
      pend = true;
      pend_par = par;
      pend_owner = owner;
      pend_lr = lr;
    }
    if (a.pivcols && me == 0 && tid == 0) a.pivcols[npiv] = (int32_t)j;
    npiv++;
    if (desc) i--; else i++;
  }
  if (a.mode == ELIM_BOTH && a.n == 0) rx = (uint32_t)i;
  // every CTA is done reading remote shared memory before anyone leaves
  cl.sync();
  if (D) {
    fold_pending();
    __syncthreads();
    cl.sync();
  }
  if (a.smem_rows) {
    for (uint32_t r = warp; r < nloc; r += nwarps) {
      const uint32_t p = pos[r];
      for (uint32_t w = lane; w < W; w += 32) {
        a.xzs[(size_t)p * W + w] = rowsbuf[(size_t)r * WS + w];
        if (D) a.dxzs[(size_t)p * W + w] = drows[(size_t)r * WS + w];
      }
      if (lane == 0 && a.phases) {
        a.ph[p] = lph[r];
        if (D) a.dph[p] = dlph[r];
      }
    }
  } else {
    for (uint32_t r = warp; r < nloc; r += nwarps) {
      const uint32_t p = pos[r];
      for (uint32_t w = lane; w < W; w += 32) {
        a.gtmp[(size_t)p * W + w] = a.xzs[(size_t)(r0 + r) * W + w];
        if (D) a.gtmp[(size_t)(a.rows + p) * W + w] = a.dxzs[(size_t)(r0 + r) * W + w];
      }
      if (lane == 0) {
        a.gtmp_ph[p] = a.phases ? lph[r] : a.ph[p];
        if (D) a.gtmp_ph[a.rows + p] = a.phases ? dlph[r] : a.dph[p];
      }
    }
  }
  if (me == 0 && tid == 0) {
    a.out[0] = (int32_t)(a.mode == ELIM_BOTH ? rx : npiv);
    a.out[1] = i;
  }
}

template <bool D, bool DESC>
__global__ void __launch_bounds__(CANON_THREADS) canon_kernel(const CanonArgs a) {
  extern __shared__ __align__(16) uint64_t smem[];
  canon_body<D, DESC>(a, smem);
}

// permutesystems!(s, perm) (src/linalg.jl:7-17): every row becomes row[perm]
// (new qubit j is old qubit perm[j], 0-based here); phases stay.  One warp per
// row, the old row staged in shared memory.
__global__ void permute_kernel(uint64_t* xzs, uint32_t rows, uint32_t n, uint32_t W, const uint32_t* perm) {
  extern __shared__ __align__(16) uint64_t pbuf[];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t len = W / 2;
  uint64_t* old = pbuf + (size_t)warp * W;
  for (uint32_t m = blockIdx.x * nw + warp; m < rows; m += gridDim.x * nw) {
    uint64_t* row = xzs + (size_t)m * W;
    for (uint32_t w = lane; w < W; w += 32) old[w] = row[w];
    __syncwarp();
    for (uint32_t w = lane; w < len; w += 32) {
      uint64_t x = 0, z = 0;
      for (uint32_t b = 0; b < 64; b++) {
        const uint32_t j = w * 64 + b;
        if (j >= n) break;
        const uint32_t q = perm[j];
        x |= ((old[q >> 6] >> (q & 63)) & 1ull) << b;
        z |= ((old[len + (q >> 6)] >> (q & 63)) & 1ull) << b;
      }
      row[w] = x;
      row[len + w] = z;
    }
    __syncwarp();
  }
}

// generate! (src/project_trace_reset.jl:41-81) on a canonical stabilizer,
// one CTA.  The Pauli lives in shared memory; each step finds the first set
// bit, the first usable row with that bit, and multiplies.
__global__ void __launch_bounds__(1024) generate_kernel(uint64_t* pauli, uint8_t* pph,
                                                        const uint64_t* xzs, const uint8_t* ph,
                                                        uint32_t rows, uint32_t W, int phases,
                                                        int32_t* ok, int32_t* used, uint32_t cap,
                                                        uint32_t* n_used) {
  extern __shared__ __align__(16) uint64_t gs[];
  uint64_t* p = gs;
  __shared__ uint32_t red[32];
  __shared__ uint32_t sh[4];
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const uint32_t len = W / 2;
  for (uint32_t w = tid; w < W; w += blockDim.x) p[w] = pauli[w];
  if (tid == 0) { sh[2] = pph[0]; sh[3] = 0; }
  __syncthreads();
  uint32_t u = 0, nu = 0, good = 1;
  for (uint32_t stage = 0; stage < 2 && good; stage++) {
    while (true) {
      // first set bit of this half
      uint32_t fb = 0xFFFFFFFFu;
      for (uint32_t w = tid; w < len; w += blockDim.x) {
        const uint64_t v = p[stage * len + w];
        if (v) fb = min(fb, w * 64 + (uint32_t)(__ffsll((long long)v) - 1));
      }
      fb = __reduce_min_sync(0xFFFFFFFFu, fb);
      if (lane == 0) red[warp] = fb;
      __syncthreads();
      if (warp == 0) {
        uint32_t b = lane < nwarps ? red[lane] : 0xFFFFFFFFu;
        b = __reduce_min_sync(0xFFFFFFFFu, b);
        if (lane == 0) sh[0] = b;
      }
      __syncthreads();
      const uint32_t bit = sh[0];
      if (bit == 0xFFFFFFFFu) break;
      const uint32_t ib = stage * len + (bit >> 6);
      const uint64_t m = 1ull << (bit & 63);
      uint32_t cand = 0xFFFFFFFFu;
      for (uint32_t r = u + tid; r < rows; r += blockDim.x)
        if (xzs[(size_t)r * W + ib] & m) { cand = min(cand, r); break; }
      cand = __reduce_min_sync(0xFFFFFFFFu, cand);
      __syncthreads();
      if (lane == 0) red[warp] = cand;
      __syncthreads();
      if (warp == 0) {
        uint32_t b = lane < nwarps ? red[lane] : 0xFFFFFFFFu;
        b = __reduce_min_sync(0xFFFFFFFFu, b);
        if (lane == 0) sh[1] = b;
      }
      __syncthreads();
      const uint32_t c = sh[1];
      if (c == 0xFFFFFFFFu) { good = 0; break; }
      u = c + 1;
      if (tid == 0 && used && nu < cap) used[nu] = (int32_t)u;
      nu++;
      if (warp == 0) {
        uint64_t c1 = 0, c2 = 0;
        const uint64_t* l = xzs + (size_t)c * W;
        for (uint32_t w = lane; w < len; w += 32) {
          uint64_t x2 = p[w], z2 = p[len + w];
          mul_step_c(l[w], l[len + w], x2, z2, c1, c2);
          p[w] = x2;
          p[len + w] = z2;
        }
        if (phases) {
          const uint32_t s =
              __reduce_add_sync(0xFFFFFFFFu, (uint32_t)(__popcll(c1) + 2 * __popcll(c2)) & 3u) & 3u;
          if (lane == 0) sh[2] = (s + sh[2] + ph[c]) & 3u;
        }
      }
      __syncthreads();
    }
  }
  // the Pauli must now be the identity up to a phase
  uint32_t nz = 0;
  for (uint32_t w = tid; w < W; w += blockDim.x) nz |= p[w] != 0;
  nz = __reduce_or_sync(0xFFFFFFFFu, nz);
  if (lane == 0) red[warp] = nz;
  __syncthreads();
  if (tid == 0) {
    uint32_t any = 0;
    for (uint32_t k = 0; k < nwarps; k++) any |= red[k];
    ok[0] = (good && !any) ? 1 : 0;
    n_used[0] = nu;
    pph[0] = (uint8_t)sh[2];
  }
  for (uint32_t w = tid; w < W; w += blockDim.x) pauli[w] = p[w];
}

// ---------------------------------------------------------------------------
// Blocked canonicalize! (X stage then Z stage, no destabilizer rows): the
// columns are taken in panels of 64.  Per panel:
//   1. after a cluster barrier every CTA gathers the panel's word of every
//      row (its own rows from shared memory, the others' through distributed
//      shared memory) and runs the panel's pivot steps on those words alone,
//      redundantly in every CTA, so the pivot search needs no cluster
//      barrier: per column the first row at position >= i with the bit, a
//      logical row swap, and the panel word of every other row with the bit
//      XORed with the pivot's.  Each row also keeps which of the panel's
//      pivot rows (as they were at the panel start) it has absorbed (a
//      64-bit mask), and each step records the pivot's mask A_t and panel
//      word;
//   2. every CTA fetches the panel's pivot rows as they were at the panel
//      start (full rows) and their phases;
//   3. after a second cluster barrier every CTA applies the panel to its own
//      rows: a row's final bits are its start bits XOR the pivot rows of its
//      mask, and its phase is replayed exactly.  With q = phase + |x & z|
//      (mod 4) a product L*R has q = q_L + q_R + 2 (z_L . x_R), and z_L . x_R
//      of two XOR-combinations of start rows is a bilinear form: with
//      C[a][b] = z_a . x_b over the pivot rows and u_m[a] = z_a . x_m,
//      z_pivot . x_m = parity(D_t & mask_m) ^ parity(u_m & A_t) where D_t is
//      the XOR of the C rows in A_t.  The pivots' own q at their steps come
//      from a triangular recurrence solved by one thread.
// The row products therefore equal the reference's mul_left! sequence bit
// for bit, phases included, for any rows (commuting or not).
constexpr uint32_t PANEL = 64;

struct BlockedLayout {
  size_t rows_off, po_off, xt_off, cml_off, c_off, a_off, pwp_off, d_off;  // u64 offsets
  size_t pos_off, stp_off;                                                 // u32 offsets
  size_t bt_off, qo_off, qp_off, lph_off, ql_off;                          // byte offsets
  size_t u32_base, u8_base, bytes;
};

__host__ __device__ inline BlockedLayout blocked_layout(uint32_t rows, uint32_t W, uint32_t RB, bool smem_rows) {
  BlockedLayout L{};
  size_t o = 0;
  L.rows_off = o; o += smem_rows ? (size_t)RB * (W + 1) : 0;
  L.po_off = o; o += (size_t)PANEL * W;
  L.xt_off = o; o += (size_t)PANEL * (W / 2);
  L.cml_off = o; o += RB;
  L.c_off = o; o += PANEL;
  L.a_off = o; o += PANEL;
  L.pwp_off = o; o += PANEL;
  L.d_off = o; o += PANEL;
  L.u32_base = o * 8;
  size_t u = 0;
  L.pos_off = u; u += rows;
  L.stp_off = u; u += PANEL;
  L.u8_base = L.u32_base + u * 4;
  size_t b = 0;
  L.bt_off = b; b += PANEL;
  L.qo_off = b; b += PANEL;
  L.qp_off = b; b += PANEL;
  L.lph_off = b; b += RB;
  L.ql_off = b; b += RB;
  L.bytes = (L.u8_base + b + 15) / 16 * 16;
  return L;
}

// The lane's part of u[x] = z_x . x_row for one row and the T pivot rows PO
// ([T][W] in shared memory): the row's X words wb + lane + 32 k, k < K
// (those below len), against pivot x's Z words, as bit x of lo (x < 32) or
// hi; s gets the lane's |x & z| of those words.  The products of a pivot's
// words are XOR-accumulated and counted once (the parity of a sum of
// popcounts is the parity of the XOR); a lane past len reads word 0 against
// a zero word, so the pivot loop has no branch.
template <int K>
__device__ __forceinline__ void row_parities(const uint64_t* PO, uint32_t W, uint32_t len, uint32_t T,
                                             uint32_t wb, uint32_t lane, const uint64_t* row, uint32_t& lo,
                                             uint32_t& hi, uint32_t& s) {
  uint64_t xw[K];
  uint32_t off[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    const uint32_t w = wb + lane + 32u * k;
    const bool ok = w < len;
    off[k] = ok ? w : 0u;
    xw[k] = ok ? row[w] : 0ull;
    if (ok) s += __popcll(xw[k] & row[len + w]);
  }
  const uint64_t* pz = PO + len;
  const uint32_t t0 = min(T, 32u);
#pragma unroll 4
  for (uint32_t x = 0; x < t0; x++) {
    uint64_t acc = 0;
#pragma unroll
    for (int k = 0; k < K; k++) acc ^= pz[(size_t)x * W + off[k]] & xw[k];
    lo ^= ((uint32_t)__popc((uint32_t)acc ^ (uint32_t)(acc >> 32)) & 1u) << x;
  }
#pragma unroll 4
  for (uint32_t x = 32; x < T; x++) {
    uint64_t acc = 0;
#pragma unroll
    for (int k = 0; k < K; k++) acc ^= pz[(size_t)x * W + off[k]] & xw[k];
    hi ^= ((uint32_t)__popc((uint32_t)acc ^ (uint32_t)(acc >> 32)) & 1u) << (x - 32);
  }
}

template <uint32_t RPT>
__device__ __forceinline__ void blocked_body(const CanonArgs& a, uint64_t* smem) {
  cg::cluster_group cl = cg::this_cluster();
  const uint32_t me = cl.block_rank();
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5, bd = blockDim.x;
  const uint32_t R = a.rows, n = a.n, W = a.W, len = W / 2, WS = W + 1, RB = a.RB;
  const uint32_t r0 = me * RB;
  const uint32_t nloc = r0 < R ? min(RB, R - r0) : 0u;
  const BlockedLayout Lo = blocked_layout(R, W, RB, a.smem_rows != 0);
  uint64_t* rowsbuf = smem + Lo.rows_off;
  uint64_t* PO = smem + Lo.po_off;
  uint64_t* XT = smem + Lo.xt_off;   // XT[w * PANEL + t] = X word w of pivot row t
  uint64_t* cml = smem + Lo.cml_off; // per local row: its mask of pivot rows in this panel
  uint64_t* C = smem + Lo.c_off;
  uint64_t* A = smem + Lo.a_off;
  uint64_t* PWP = smem + Lo.pwp_off;
  uint64_t* Dt = smem + Lo.d_off;
  uint32_t* u32b = (uint32_t*)((uint8_t*)smem + Lo.u32_base);
  uint32_t* pos = u32b + Lo.pos_off;
  uint32_t* stp = u32b + Lo.stp_off;
  uint8_t* u8b = (uint8_t*)smem + Lo.u8_base;
  uint8_t* bt = u8b + Lo.bt_off;
  uint8_t* qo = u8b + Lo.qo_off;
  uint8_t* qp = u8b + Lo.qp_off;
  uint8_t* lph = u8b + Lo.lph_off;
  uint8_t* ql = u8b + Lo.ql_off;     // per local row: its q after the panel

  // per search warp and column parity: its best (position << 32 | row), that
  // row's panel word and mask
  __shared__ uint64_t red2[2][32][3];
  __shared__ uint32_t shT, shI;     // the search warps' step count and next position
  __shared__ uint64_t Us[PANEL];   // pivot t's updates before its own step
  __shared__ uint8_t bases[PANEL];
  auto ROW = [&](uint32_t lr) -> uint64_t* {
    return a.smem_rows ? rowsbuf + (size_t)lr * WS : a.xzs + (size_t)(r0 + lr) * W;
  };
  // word w of physical row r, wherever it lives
  auto RWORD = [&](uint32_t r, uint32_t w) -> uint64_t {
    if (!a.smem_rows) return a.xzs[(size_t)r * W + w];
    const uint32_t o = r / RB, lr = r - o * RB;
    const uint64_t* src = rowsbuf + (size_t)lr * WS + w;
    return o == me ? *src : *cl.map_shared_rank(src, o);
  };

  for (uint32_t lr = tid; lr < nloc; lr += bd) lph[lr] = a.ph[r0 + lr];
  if (a.smem_rows)
    for (uint32_t lr = warp; lr < nloc; lr += nwarps)
      for (uint32_t w = lane; w < W; w += 32) rowsbuf[(size_t)lr * WS + w] = a.xzs[(size_t)(r0 + lr) * W + w];
  // the panel's pivot search runs on the first NB warps only, each thread
  // owning rows tid, tid + nbt, ... (at most RPT) whose positions, panel
  // words and masks it keeps in registers; named barrier 1 synchronises them
  const uint32_t NB = min(nwarps, max(1u, (R + 32 * RPT - 1) / (32 * RPT))), nbt = NB * 32;
  uint32_t rpos[RPT];
  uint64_t rpw[RPT], rcb[RPT];
#pragma unroll
  for (uint32_t k = 0; k < RPT; k++) { rpos[k] = tid + k * nbt; rpw[k] = 0; rcb[k] = 0; }

  uint32_t i = 0, rx = 0;
  for (uint32_t stage = 0; stage < 2; stage++) {
    for (uint32_t c0 = 0; c0 < n && i < R; c0 += PANEL) {
      const uint32_t ncp = min(PANEL, n - c0), wj = stage * len + (c0 >> 6);
      cl.sync();  // every row is final for this panel (and every CTA is done with the last one)
      // ---- 1. the panel words of all rows; the panel's pivot steps
      if (warp < NB) {
#pragma unroll
        for (uint32_t k = 0; k < RPT; k++) {
          const uint32_t r = tid + k * nbt;
          rpw[k] = r < R ? RWORD(r, wj) : 0ull;
          rcb[k] = 0;
        }
      }
      // One block barrier per column: every thread evaluates its rows (after
      // applying the previous step to them), each warp publishes its best
      // (position, row), and after the barrier every warp reduces the
      // published pairs itself.  Each row's owner thread moves its own row
      // (pos[] is per row, nothing else tracks positions); the pivot's owner
      // records the step for the panel application.
      uint32_t T = 0;
      if (warp < NB) {
        bool prev = false;
        uint32_t pprev = 0, bprev = 0;
        uint64_t pwprev = 0, aprev = 0;
        for (uint32_t b = 0; b < ncp && i < R; b++) {
          uint32_t bpos = 0xFFFFFFFFu, bk = 0;
#pragma unroll
          for (uint32_t k = 0; k < RPT; k++) {
            const uint32_t r = tid + k * nbt;
            if (r >= R) continue;
            if (prev && r != pprev && ((rpw[k] >> bprev) & 1ull)) {  // the previous step's elimination
              rpw[k] ^= pwprev;
              rcb[k] ^= aprev;
            }
            if (rpos[k] >= i && ((rpw[k] >> b) & 1ull) && rpos[k] < bpos) { bpos = rpos[k]; bk = k; }
          }
          {
            uint64_t mypw = 0, mycb = 0;
#pragma unroll
            for (uint32_t k = 0; k < RPT; k++)
              if (k == bk) { mypw = rpw[k]; mycb = rcb[k]; }
            const uint32_t m = __reduce_min_sync(0xFFFFFFFFu, bpos);
            const uint32_t who = __ballot_sync(0xFFFFFFFFu, bpos == m);
            const uint32_t src = __ffs(who) - 1;
            const uint32_t row = __shfl_sync(0xFFFFFFFFu, tid + bk * nbt, src);
            const uint64_t wpw = __shfl_sync(0xFFFFFFFFu, mypw, src);
            const uint64_t wcb = __shfl_sync(0xFFFFFFFFu, mycb, src);
            if (lane == 0) {
              red2[b & 1][warp][0] = ((uint64_t)m << 32) | row;
              red2[b & 1][warp][1] = wpw;
              red2[b & 1][warp][2] = wcb;
            }
          }
          // the only barrier of the column: the buffer of column b + 2 is
          // written after every search warp has passed the barrier of b + 1
          asm volatile("bar.sync 1, %0;" ::"r"(nbt) : "memory");
          const uint64_t e = lane < NB ? red2[b & 1][lane][0] : ~0ull;
          const uint32_t kpos = __reduce_min_sync(0xFFFFFFFFu, (uint32_t)(e >> 32));
          if (kpos == 0xFFFFFFFFu) {  // no row has the bit: no pivot in this column
            prev = false;
            continue;
          }
          const uint32_t kw = __ffs(__ballot_sync(0xFFFFFFFFu, (uint32_t)(e >> 32) == kpos)) - 1;
          const uint32_t pstar = (uint32_t)red2[b & 1][kw][0];
          pwprev = red2[b & 1][kw][1];
          aprev = red2[b & 1][kw][2] | (1ull << T);
          // rowswap!(state, k, i): the rows at positions kpos and i trade places
#pragma unroll
          for (uint32_t k = 0; k < RPT; k++) {
            const uint32_t r = tid + k * nbt;
            if (r == pstar) rpos[k] = i;
            else if (r < R && rpos[k] == i) rpos[k] = kpos;
          }
          if (tid == 0) {
            stp[T] = pstar;
            bt[T] = (uint8_t)b;
            A[T] = aprev;
            PWP[T] = pwprev;
          }
          prev = true;
          pprev = pstar;
          bprev = b;
          T++;
          i++;
        }
        if (tid == 0) { shT = T; shI = i; }
      }
      __syncthreads();  // the step records and the last positions are written
      T = shT;
      i = shI;
      if (T == 0) continue;  // no pivot in this panel: nothing to apply
      // ---- 2. the pivot rows as they were at the panel start, their q
      for (uint32_t t = warp; t < T; t += nwarps) {
        const uint32_t r = stp[t];
        uint32_t s = 0;
        for (uint32_t w = lane; w < W; w += 32) {
          const uint64_t v = RWORD(r, w);
          PO[(size_t)t * W + w] = v;
          if (w < len) XT[(size_t)w * PANEL + t] = v;
        }
        __syncwarp();
        for (uint32_t w = lane; w < len; w += 32) s += __popcll(PO[(size_t)t * W + w] & PO[(size_t)t * W + len + w]);
        s = __reduce_add_sync(0xFFFFFFFFu, s);
        if (lane == 0) {
          const uint32_t o = r / RB, lr = r - o * RB;
          const uint8_t ph0 = o == me ? lph[lr] : *cl.map_shared_rank(lph + lr, o);
          qo[t] = (uint8_t)((ph0 + s) & 3u);
        }
      }
      __syncthreads();
      // C[a] bit b = z_a . x_b over the pivot rows: lane b reads the
      // transposed X words (conflict-free), z_a is a broadcast
      for (uint32_t t = warp; t < T; t += nwarps) {
        const uint64_t* za = PO + (size_t)t * W + len;
        uint64_t p0 = 0, p1 = 0;  // XOR-accumulated: the parity is the popcount's
        for (uint32_t w = 0; w < len; w++) {
          const uint64_t zw = za[w];
          p0 ^= zw & XT[(size_t)w * PANEL + lane];
          p1 ^= zw & XT[(size_t)w * PANEL + lane + 32];
        }
        const uint32_t lo = __ballot_sync(0xFFFFFFFFu, (__popcll(p0) & 1) && lane < T);
        const uint32_t hi = __ballot_sync(0xFFFFFFFFu, (__popcll(p1) & 1) && lane + 32 < T);
        if (lane == 0) C[t] = (uint64_t)lo | ((uint64_t)hi << 32);
      }
      __syncthreads();
      if (a.phases) {
        // D_t = XOR of the C rows in A_t; then for each pivot its updates
        // before its own step give q_t = base_t + (sum of q_t' over them)
        if (tid < T) {
          uint64_t d = 0;
          for (uint32_t x = 0; x < T; x++)
            if ((A[tid] >> x) & 1ull) d ^= C[x];
          Dt[tid] = d;
        }
        __syncthreads();
        if (tid < T) {
          const uint32_t t = tid;
          uint64_t u = 0;  // u[x] = z_x . x_(pivot t) = C[x] bit t
          for (uint32_t x = 0; x < T; x++) u |= ((C[x] >> t) & 1ull) << x;
          uint64_t pw = PO[(size_t)t * W + wj], cm = 0, ut = 0;
          uint32_t cross = 0;
          for (uint32_t t2 = 0; t2 < t; t2++) {
            if ((pw >> bt[t2]) & 1ull) {
              cross += (uint32_t)((__popcll(Dt[t2] & cm) + __popcll(u & A[t2])) & 1);
              ut |= 1ull << t2;
              cm ^= A[t2];
              pw ^= PWP[t2];
            }
          }
          Us[t] = ut;
          bases[t] = (uint8_t)((qo[t] + 2u * cross) & 3u);
        }
        __syncthreads();
        if (tid == 0) {
          uint64_t Q1 = 0, Q2 = 0;  // bit t: bit 0 / bit 1 of q_t
          for (uint32_t t = 0; t < T; t++) {
            const uint32_t q = (bases[t] + (uint32_t)__popcll(Us[t] & Q1) + 2u * (uint32_t)__popcll(Us[t] & Q2)) & 3u;
            qp[t] = (uint8_t)q;
            Q1 |= (uint64_t)(q & 1u) << t;
            Q2 |= (uint64_t)(q >> 1) << t;
          }
        }
      }
      cl.sync();  // every CTA is done reading other CTAs' rows
      // ---- 3. the panel applied to the local rows
      // (a) per row (warp per row): u[x] = z_x . x_row and q = phase + |x & z|
      if (a.phases) {
        for (uint32_t lr = warp; lr < nloc; lr += nwarps) {
          const uint64_t* row = ROW(lr);
          uint32_t lo = 0, hi = 0, s = 0;
          for (uint32_t wb = 0; wb < len; wb += 128) {
            const uint32_t kn = min(4u, (len - wb + 31) / 32);  // warp-uniform
            if (kn == 1) row_parities<1>(PO, W, len, T, wb, lane, row, lo, hi, s);
            else if (kn == 2) row_parities<2>(PO, W, len, T, wb, lane, row, lo, hi, s);
            else if (kn == 3) row_parities<3>(PO, W, len, T, wb, lane, row, lo, hi, s);
            else row_parities<4>(PO, W, len, T, wb, lane, row, lo, hi, s);
          }
          s = __reduce_add_sync(0xFFFFFFFFu, s);
          lo = __reduce_xor_sync(0xFFFFFFFFu, lo);
          hi = __reduce_xor_sync(0xFFFFFFFFu, hi);
          if (lane == 0) {
            cml[lr] = (uint64_t)lo | ((uint64_t)hi << 32);
            ql[lr] = (uint8_t)((lph[lr] + s) & 3u);
          }
        }
        __syncthreads();
      }
      // (b) the steps replayed, one thread per row: its mask and its q
      for (uint32_t lr = tid; lr < nloc; lr += bd) {
        const uint32_t r = r0 + lr;
        uint64_t pw = ROW(lr)[wj], cm = 0;
        const uint64_t u = a.phases ? cml[lr] : 0;
        uint32_t q = a.phases ? ql[lr] : 0;
        for (uint32_t t = 0; t < T; t++) {
          if (r != stp[t] && ((pw >> bt[t]) & 1ull)) {
            if (a.phases) q += qp[t] + 2u * (uint32_t)((__popcll(Dt[t] & cm) + __popcll(u & A[t])) & 1);
            cm ^= A[t];
            pw ^= PWP[t];
          }
        }
        cml[lr] = cm;
        ql[lr] = (uint8_t)(q & 3u);
      }
      __syncthreads();
      // (c) the rows (warp per row): start bits XOR the pivot rows of the mask
      for (uint32_t lr = warp; lr < nloc; lr += nwarps) {
        const uint64_t cm = cml[lr];
        if (!cm) continue;
        uint64_t* row = ROW(lr);
        uint32_t s = 0;
        for (uint32_t w = lane; w < len; w += 32) {
          uint64_t vx = row[w], vz = row[len + w];
          uint64_t m = cm;
          while (m) {
            const uint32_t x = __ffsll(m) - 1;
            m &= m - 1;
            vx ^= PO[(size_t)x * W + w];
            vz ^= PO[(size_t)x * W + len + w];
          }
          row[w] = vx;
          row[len + w] = vz;
          s += __popcll(vx & vz);
        }
        if (a.phases) {
          s = __reduce_add_sync(0xFFFFFFFFu, s);
          if (lane == 0) lph[lr] = (uint8_t)((ql[lr] - s) & 3u);
        }
      }
    }
    if (stage == 0) rx = i;
  }
  if (warp < NB) {
#pragma unroll
    for (uint32_t k = 0; k < RPT; k++)
      if (tid + k * nbt < R) pos[tid + k * nbt] = rpos[k];
  }
  __syncthreads();
  cl.sync();
  // rows to their final positions
  if (a.smem_rows) {
    for (uint32_t lr = warp; lr < nloc; lr += nwarps) {
      const uint32_t p = pos[r0 + lr];
      for (uint32_t w = lane; w < W; w += 32) a.xzs[(size_t)p * W + w] = rowsbuf[(size_t)lr * WS + w];
      if (lane == 0 && a.phases) a.ph[p] = lph[lr];
    }
  } else {
    for (uint32_t lr = warp; lr < nloc; lr += nwarps) {
      const uint32_t p = pos[r0 + lr];
      for (uint32_t w = lane; w < W; w += 32) a.gtmp[(size_t)p * W + w] = a.xzs[(size_t)(r0 + lr) * W + w];
      if (lane == 0) a.gtmp_ph[p] = a.phases ? lph[lr] : a.ph[p];
    }
    if (a.copy_back) {
      // every CTA has written its rows to their final places in gtmp
      cl.sync();
      for (uint32_t lr = warp; lr < nloc; lr += nwarps) {
        const uint32_t r = r0 + lr;
        for (uint32_t w = lane; w < W; w += 32) a.xzs[(size_t)r * W + w] = a.gtmp[(size_t)r * W + w];
        if (lane == 0) a.ph[r] = a.gtmp_ph[r];
      }
    }
  }
  if (me == 0 && tid == 0) {
    a.out[0] = (int32_t)rx;
    a.out[1] = (int32_t)i;
  }
}

template <uint32_t RPT>
__global__ void __launch_bounds__(CANON_THREADS) canon_blocked_kernel(const CanonArgs a) {
  extern __shared__ __align__(16) uint64_t smem[];
  blocked_body<RPT>(a, smem);
}

// Many canonicalize! jobs (stabilizer tableaux) drained by persistent
// clusters: CTA 0 of a cluster takes the next job from the queue (longest
// first) and the cluster runs it (by panels, or by column steps), then the
// next.  The job's arguments are copied into shared memory.
struct CanonBatchArgs {
  const CanonArgs* jobs;
  uint32_t njobs;
  uint32_t* head;  // next job (zero before the launch)
  int blocked;     // 1: the jobs run by panels (blocked_body), else by column steps
};
static_assert(sizeof(CanonArgs) % 8 == 0, "CanonArgs is copied in 8-byte words");

__global__ void __launch_bounds__(CANON_THREADS) canon_batch_kernel(const CanonBatchArgs b) {
  extern __shared__ __align__(16) uint64_t smem[];
  __shared__ __align__(16) CanonArgs ja;
  __shared__ uint32_t jobid;
  cg::cluster_group cl = cg::this_cluster();
  const uint32_t me = cl.block_rank(), tid = threadIdx.x;
  while (true) {
    if (me == 0 && tid == 0) {
      const uint32_t j = atomicAdd(b.head, 1u);
      jobid = j < b.njobs ? j : 0xFFFFFFFFu;
    }
    cl.sync();
    const uint32_t j = *cl.map_shared_rank(&jobid, 0);
    if (j == 0xFFFFFFFFu) break;
    for (uint32_t w = tid; w < sizeof(CanonArgs) / 8; w += blockDim.x)
      ((uint64_t*)&ja)[w] = ((const uint64_t*)(b.jobs + j))[w];
    __syncthreads();
    if (b.blocked) blocked_body<4>(ja, smem);
    else canon_body<false, false>(ja, smem);
    __syncthreads();  // ja is read until the end of the body
  }
  cl.sync();  // CTA 0's job slot is read by the cluster until here
}

// ---------------------------------------------------------------- panels over the whole GPU
// canonicalize! by 64-column panels with the per-row work spread over every
// SM: per panel two launches, (1) canon_search_kernel, one CTA: the panel's
// pivot steps on the panel words of all rows (the same search as
// blocked_body, positions kept in global memory between panels), the pivot
// rows as they are at the panel start copied aside, and the panel's phase
// data (C, D_t, the pivots' q); (2) canon_apply_kernel, a grid over the rows:
// every row's mask, bits and phase from that record (the same bilinear-form
// replay as blocked_body).  The launch boundary is the barrier between the
// two; the rows live in global memory (L2-resident) throughout.
struct PanelRec {
  uint32_t T;        // pivots of the panel
  uint32_t i;        // next pivot position after the panel
  uint32_t rx;       // pivots of the X stage (kept from the last X-stage panel)
  uint32_t done;     // every position has a pivot: later panels do nothing
  uint32_t stp[PANEL];
  uint8_t bt[PANEL];
  uint8_t qp[PANEL];
  uint64_t A[PANEL], PWP[PANEL], Dt[PANEL];
};

struct PanelArgs {
  uint64_t* xzs;
  uint8_t* ph;
  uint32_t rows, n, W;
  int phases;
  uint32_t stage, c0;   // this panel: stage 0 (X) or 1 (Z), first column
  uint32_t* pos;        // [rows] row -> position (persistent)
  PanelRec* rec;        // this panel's record
  uint64_t* po;         // [PANEL][W] the pivot rows at the panel start
  int32_t* out;         // [0] X-stage pivots, [1] next pivot position
  // look-ahead schedule only
  PanelRec* prev;       // the previous panel's record (its i / rx / done start this panel)
  uint64_t* po_prev;    // the previous panel's pivot rows
  uint64_t* nw;         // [rows] each row's word of this panel (of the next one, once written)
  uint32_t wj_prev;     // word index of the previous panel (UINT32_MAX: none)
  uint32_t wj_next;     // word index of the next panel (UINT32_MAX: none)
  uint32_t steps;       // 1: this launch runs this panel's pivot steps
};

// The word index of a panel's columns in a row (X words, then Z words).
__host__ __device__ inline uint32_t panel_word(uint32_t stage, uint32_t c0, uint32_t len) {
  return stage * len + (c0 >> 6);
}

// (1) The panel's pivot steps on the panel words of the candidate rows
// (positions >= the next pivot position), word(r) = wsrc[r * wstride]; the
// positions of those rows are updated in `pos`, and the record g gets the
// pivot rows, their columns, masks and words (stp, bt, A, PWP) and T, i, rx,
// done, starting from prev's i / rx / done (prev may be g itself).
template <uint32_t RPT>
__device__ __forceinline__ void panel_steps(const PanelArgs& a, const PanelRec& prev, PanelRec& g,
                                            const uint64_t* wsrc, uint32_t wstride, uint32_t* cand) {
  __shared__ uint32_t stp[PANEL];
  __shared__ uint8_t bt[PANEL];
  __shared__ uint64_t A[PANEL], PWP[PANEL];
  __shared__ uint64_t red2[2][32][3];
  __shared__ uint32_t shT, shI, ncand;
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const uint32_t R = a.rows, n = a.n;
  const uint32_t c0 = a.c0, ncp = min(PANEL, n - c0);
  uint32_t i = prev.i;
  const uint32_t rx0 = prev.rx;
  if (prev.done) {  // every position has its pivot: this panel applies nothing
    __syncthreads();  // every thread has read prev before g (maybe prev) is written
    if (tid == 0) { g.T = 0; g.i = i; g.rx = rx0; g.done = 1; }
    __syncthreads();
    return;
  }
  // Only rows at positions >= i can become pivots; the search runs on them
  // alone (the others' panel words do not matter to it), so it shrinks as
  // the elimination proceeds.
  if (tid == 0) ncand = 0;
  __syncthreads();
  for (uint32_t r = tid; r < R; r += blockDim.x)
    if (a.pos[r] >= i) cand[atomicAdd(&ncand, 1u)] = r;
  __syncthreads();
  const uint32_t Rc = ncand;
  const uint32_t NB = min(nwarps, max(1u, (Rc + 32 * RPT - 1) / (32 * RPT))), nbt = NB * 32;
  uint32_t rrow[RPT], rpos[RPT];
  uint64_t rpw[RPT], rcb[RPT];
  uint32_t T = 0;
  if (warp < NB) {
#pragma unroll
    for (uint32_t k = 0; k < RPT; k++) {
      const uint32_t j = tid + k * nbt;
      rrow[k] = j < Rc ? cand[j] : 0xFFFFFFFFu;
      rpos[k] = j < Rc ? a.pos[rrow[k]] : 0xFFFFFFFFu;
      rpw[k] = j < Rc ? wsrc[(size_t)rrow[k] * wstride] : 0ull;
      rcb[k] = 0;
    }
    // the steps (as blocked_body): one named barrier among the search warps
    // per column.  Kept short, as the search is instruction-bound on its SM:
    // rows past the candidates hold a zero word (never a candidate, never
    // updated); the previous step's pivot is applied lazily at the start of
    // a step (pwprev = 0 after a column without one), which also zeroes the
    // pivot row's own word, so it never competes again; positions i and kpos
    // swap by value; the warp's best row travels with its position and the
    // winning lane posts it.
    uint32_t bprev = 0;
    uint64_t pwprev = 0, aprev = 0;
    for (uint32_t b = 0; b < ncp && i < R; b++) {
      uint32_t bpos = 0xFFFFFFFFu, brow = 0;
      uint64_t bpw = 0, bcb = 0;
#pragma unroll
      for (uint32_t k = 0; k < RPT; k++) {
        if ((rpw[k] >> bprev) & 1ull) {
          rpw[k] ^= pwprev;
          rcb[k] ^= aprev;
        }
        if (((rpw[k] >> b) & 1ull) && rpos[k] < bpos) {
          bpos = rpos[k];
          brow = rrow[k];
          bpw = rpw[k];
          bcb = rcb[k];
        }
      }
      {
        const uint32_t m = __reduce_min_sync(0xFFFFFFFFu, bpos);
        const uint32_t src = __ffs(__ballot_sync(0xFFFFFFFFu, bpos == m)) - 1;
        if (lane == src) {
          red2[b & 1][warp][0] = ((uint64_t)m << 32) | brow;
          red2[b & 1][warp][1] = bpw;
          red2[b & 1][warp][2] = bcb;
        }
      }
      asm volatile("bar.sync 1, %0;" ::"r"(nbt) : "memory");
      const uint64_t e = lane < NB ? red2[b & 1][lane][0] : ~0ull;
      const uint32_t kpos = __reduce_min_sync(0xFFFFFFFFu, (uint32_t)(e >> 32));
      if (kpos == 0xFFFFFFFFu) {
        pwprev = 0;
        aprev = 0;
        continue;
      }
      const uint32_t kw = __ffs(__ballot_sync(0xFFFFFFFFu, (uint32_t)(e >> 32) == kpos)) - 1;
      pwprev = red2[b & 1][kw][1];
      aprev = red2[b & 1][kw][2] | (1ull << T);
#pragma unroll
      for (uint32_t k = 0; k < RPT; k++) rpos[k] = rpos[k] == kpos ? i : (rpos[k] == i ? kpos : rpos[k]);
      if (tid == 0) {
        stp[T] = (uint32_t)red2[b & 1][kw][0];
        bt[T] = (uint8_t)b;
        A[T] = aprev;
        PWP[T] = pwprev;
      }
      bprev = b;
      T++;
      i++;
    }
#pragma unroll
    for (uint32_t k = 0; k < RPT; k++)
      if (rrow[k] != 0xFFFFFFFFu) a.pos[rrow[k]] = rpos[k];
    if (tid == 0) { shT = T; shI = i; }
  }
  __syncthreads();
  T = shT;
  i = shI;
  for (uint32_t t = tid; t < T; t += blockDim.x) {
    g.stp[t] = stp[t];
    g.bt[t] = bt[t];
    g.A[t] = A[t];
    g.PWP[t] = PWP[t];
  }
  if (tid == 0) {
    g.T = T;
    g.i = i;
    g.rx = a.stage == 0 ? i : rx0;
    g.done = i >= R ? 1u : 0u;
    a.out[0] = (int32_t)g.rx;
    a.out[1] = (int32_t)i;
  }
  __syncthreads();  // the record is complete for the whole CTA
}

// (2) The pivot rows of the record g as they are at the panel start: copied
// to po, their q = phase + |x & z|, and the panel's phase data (C, D_t and
// the pivots' q, into g.Dt and g.qp).  wj: the panel's word index.
__device__ __forceinline__ void panel_post(const PanelArgs& a, PanelRec& g, uint64_t* po, uint32_t wj,
                                           uint64_t* XT) {
  __shared__ uint32_t stp[PANEL];
  __shared__ uint8_t bt[PANEL], qo[PANEL];
  __shared__ uint64_t A[PANEL], PWP[PANEL], C[PANEL], Dt[PANEL], Us[PANEL];
  __shared__ uint8_t bases[PANEL];
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const uint32_t W = a.W, len = W / 2;
  const uint32_t T = g.T;
  // XT[w * XS + t] / ZT[w * XS + t]: X / Z word w of pivot t; the odd stride
  // keeps the transposing stores (lane = word) free of bank conflicts
  constexpr uint32_t XS = PANEL + 1;
  uint64_t* ZT = XT + (size_t)len * XS;
  for (uint32_t t = tid; t < T; t += blockDim.x) {
    stp[t] = g.stp[t];
    bt[t] = g.bt[t];
    A[t] = g.A[t];
    PWP[t] = g.PWP[t];
  }
  __syncthreads();
  // the pivot rows at the panel start, their q = phase + |x & z|, XT, ZT
  for (uint32_t t = warp; t < T; t += nwarps) {
    const uint32_t r = stp[t];
    uint32_t s = 0;
    for (uint32_t w = lane; w < len; w += 32) {
      const uint64_t vx = a.xzs[(size_t)r * W + w], vz = a.xzs[(size_t)r * W + len + w];
      po[(size_t)t * W + w] = vx;
      po[(size_t)t * W + len + w] = vz;
      XT[(size_t)w * XS + t] = vx;
      ZT[(size_t)w * XS + t] = vz;
      s += __popcll(vx & vz);
    }
    s = __reduce_add_sync(0xFFFFFFFFu, s);
    if (lane == 0) qo[t] = (uint8_t)((a.ph[r] + s) & 3u);
  }
  __syncthreads();
  if (a.phases && T) {
    // C[a] bit b = z_a . x_b over the pivot rows (both transposed in shared
    // memory); the parity of a sum of popcounts is the parity of the XOR of
    // the words, so the words are XOR-accumulated and counted once
    for (uint32_t t = warp; t < T; t += nwarps) {
      uint64_t p0 = 0, p1 = 0;
      for (uint32_t w = 0; w < len; w++) {
        const uint64_t zw = ZT[(size_t)w * XS + t];
        p0 ^= zw & XT[(size_t)w * XS + lane];
        p1 ^= zw & XT[(size_t)w * XS + lane + 32];
      }
      const uint32_t lo = __ballot_sync(0xFFFFFFFFu, (__popcll(p0) & 1) && lane < T);
      const uint32_t hi = __ballot_sync(0xFFFFFFFFu, (__popcll(p1) & 1) && lane + 32 < T);
      if (lane == 0) C[t] = (uint64_t)lo | ((uint64_t)hi << 32);
    }
    __syncthreads();
    if (tid < T) {
      uint64_t d = 0;
      for (uint32_t x = 0; x < T; x++)
        if ((A[tid] >> x) & 1ull) d ^= C[x];
      Dt[tid] = d;
    }
    __syncthreads();
    if (tid < T) {
      const uint32_t t = tid;
      uint64_t u = 0;
      for (uint32_t x = 0; x < T; x++) u |= ((C[x] >> t) & 1ull) << x;
      uint64_t pw = po[(size_t)t * W + wj], cm = 0, ut = 0;
      uint32_t cross = 0;
      for (uint32_t t2 = 0; t2 < t; t2++) {
        if ((pw >> bt[t2]) & 1ull) {
          cross += (uint32_t)((__popcll(Dt[t2] & cm) + __popcll(u & A[t2])) & 1);
          ut |= 1ull << t2;
          cm ^= A[t2];
          pw ^= PWP[t2];
        }
      }
      Us[t] = ut;
      bases[t] = (uint8_t)((qo[t] + 2u * cross) & 3u);
    }
    __syncthreads();
    if (tid == 0) {
      uint64_t Q1 = 0, Q2 = 0;
      for (uint32_t t = 0; t < T; t++) {
        const uint32_t q = (bases[t] + (uint32_t)__popcll(Us[t] & Q1) + 2u * (uint32_t)__popcll(Us[t] & Q2)) & 3u;
        g.qp[t] = (uint8_t)q;
        Q1 |= (uint64_t)(q & 1u) << t;
        Q2 |= (uint64_t)(q >> 1) << t;
      }
    }
  }
  for (uint32_t t = tid; t < T; t += blockDim.x) g.Dt[t] = a.phases ? Dt[t] : 0ull;
}

// (3) Rows of block blk of nblk: apply the record g (pivot rows po at the
// panel start, word index wj) to every row, as blocked_body's step 3 with
// rows and phases in global memory.
__device__ __forceinline__ void panel_apply(const PanelArgs& a, const PanelRec& g, const uint64_t* po,
                                            uint32_t wj, uint32_t blk, uint32_t nblk, uint64_t* sm) {
  const uint32_t T = g.T;
  if (T == 0) return;
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5, bd = blockDim.x;
  const uint32_t R = a.rows, W = a.W, len = W / 2;
  const uint32_t per = (R + nblk - 1) / nblk, r0 = blk * per;
  const uint32_t nloc = r0 < R ? min(per, R - r0) : 0u;
  if (!nloc) return;
  uint64_t* PO = sm;                      // [T][W]
  uint64_t* cml = PO + (size_t)PANEL * W; // per local row: mask
  uint8_t* ql = (uint8_t*)(cml + per);    // per local row: q
  __shared__ uint32_t stp[PANEL];
  __shared__ uint8_t bt[PANEL], qp[PANEL];
  __shared__ uint64_t A[PANEL], PWP[PANEL], Dt[PANEL];
  for (uint32_t t = tid; t < T; t += bd) {
    stp[t] = g.stp[t]; bt[t] = g.bt[t]; qp[t] = g.qp[t];
    A[t] = g.A[t]; PWP[t] = g.PWP[t]; Dt[t] = g.Dt[t];
  }
  for (size_t w = tid; w < (size_t)T * W; w += bd) PO[w] = po[w];
  __syncthreads();
  // (a) per row (warp per row): u[x] = z_x . x_row and q = phase + |x & z|;
  // the lane's X words (up to four at a time) stay in registers, and for
  // each pivot x their products with z_x are XOR-accumulated and counted
  // once (parity of the XOR = parity of the popcounts)
  if (a.phases) {
    for (uint32_t lr = warp; lr < nloc; lr += nwarps) {
      const uint64_t* row = a.xzs + (size_t)(r0 + lr) * W;
      uint32_t lo = 0, hi = 0, s = 0;
      for (uint32_t wb = 0; wb < len; wb += 128) {
        const uint32_t kn = min(4u, (len - wb + 31) / 32);  // warp-uniform
        if (kn == 1) row_parities<1>(PO, W, len, T, wb, lane, row, lo, hi, s);
        else if (kn == 2) row_parities<2>(PO, W, len, T, wb, lane, row, lo, hi, s);
        else if (kn == 3) row_parities<3>(PO, W, len, T, wb, lane, row, lo, hi, s);
        else row_parities<4>(PO, W, len, T, wb, lane, row, lo, hi, s);
      }
      s = __reduce_add_sync(0xFFFFFFFFu, s);
      lo = __reduce_xor_sync(0xFFFFFFFFu, lo);
      hi = __reduce_xor_sync(0xFFFFFFFFu, hi);
      if (lane == 0) {
        cml[lr] = (uint64_t)lo | ((uint64_t)hi << 32);
        ql[lr] = (uint8_t)((a.ph[r0 + lr] + s) & 3u);
      }
    }
    __syncthreads();
  }
  // (b) the steps replayed, one thread per row
  for (uint32_t lr = tid; lr < nloc; lr += bd) {
    const uint32_t r = r0 + lr;
    uint64_t pw = a.xzs[(size_t)r * W + wj], cm = 0;
    const uint64_t u = a.phases ? cml[lr] : 0;
    uint32_t q = a.phases ? ql[lr] : 0;
    for (uint32_t t = 0; t < T; t++) {
      if (r != stp[t] && ((pw >> bt[t]) & 1ull)) {
        if (a.phases) q += qp[t] + 2u * (uint32_t)((__popcll(Dt[t] & cm) + __popcll(u & A[t])) & 1);
        cm ^= A[t];
        pw ^= PWP[t];
      }
    }
    cml[lr] = cm;
    ql[lr] = (uint8_t)(q & 3u);
  }
  __syncthreads();
  // (c) the rows: start bits XOR the pivot rows of the mask
  for (uint32_t lr = warp; lr < nloc; lr += nwarps) {
    const uint64_t cm = cml[lr];
    if (!cm) continue;
    uint64_t* row = a.xzs + (size_t)(r0 + lr) * W;
    uint32_t s = 0;
    for (uint32_t w = lane; w < len; w += 32) {
      uint64_t vx = row[w], vz = row[len + w];
      uint64_t m = cm;
      while (m) {
        const uint32_t x = __ffsll(m) - 1;
        m &= m - 1;
        vx ^= PO[(size_t)x * W + w];
        vz ^= PO[(size_t)x * W + len + w];
      }
      row[w] = vx;
      row[len + w] = vz;
      s += __popcll(vx & vz);
    }
    if (a.phases) {
      s = __reduce_add_sync(0xFFFFFFFFu, s);
      if (lane == 0) a.ph[r0 + lr] = (uint8_t)((ql[lr] - s) & 3u);
    }
  }
}

// (4) Look-ahead: every row's word wn (the next panel's) after this panel,
// into a.nw, computed before the panel's apply has run: the row's mask by the
// same replay as the apply's step (b) on its word wj, then its word wn XOR
// the pivot rows' words wn of the mask (all read at the panel start).
__device__ __forceinline__ void panel_next(const PanelArgs& a, const PanelRec& g, uint32_t wj, uint32_t wn,
                                           uint32_t blk, uint32_t nblk) {
  __shared__ uint32_t stp[PANEL];
  __shared__ uint8_t bt[PANEL];
  __shared__ uint64_t A[PANEL], PWP[PANEL], PN[PANEL];
  const uint32_t T = g.T, tid = threadIdx.x, R = a.rows, W = a.W;
  for (uint32_t t = tid; t < T; t += blockDim.x) {
    stp[t] = g.stp[t]; bt[t] = g.bt[t]; A[t] = g.A[t]; PWP[t] = g.PWP[t];
    PN[t] = a.xzs[(size_t)g.stp[t] * W + wn];
  }
  __syncthreads();
  const uint32_t per = (R + nblk - 1) / nblk, r0 = blk * per, r1 = min(R, r0 + per);
  for (uint32_t r = r0 + tid; r < r1; r += blockDim.x) {
    uint64_t pw = a.xzs[(size_t)r * W + wj], cm = 0;
    for (uint32_t t = 0; t < T; t++) {
      if (r != stp[t] && ((pw >> bt[t]) & 1ull)) {
        cm ^= A[t];
        pw ^= PWP[t];
      }
    }
    uint64_t v = a.xzs[(size_t)r * W + wn];
    while (cm) {
      const uint32_t x = __ffsll(cm) - 1;
      cm &= cm - 1;
      v ^= PN[x];
    }
    a.nw[r] = v;
  }
}

// The plain schedule: per panel a one-CTA search launch (steps, then the
// pivot rows and phase data) and a grid-wide apply launch.
template <uint32_t RPT>
__global__ void __launch_bounds__(CANON_THREADS) canon_search_kernel(const PanelArgs a) {
  extern __shared__ __align__(16) uint64_t sm[];
  // launched as a programmatic dependent of the previous panel's apply: wait
  // for it (complete, its writes visible), then let the next launch in
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;");
  PanelRec& g = *a.rec;
  const uint32_t len = a.W / 2, wj = panel_word(a.stage, a.c0, len);
  uint64_t* XT = sm;                                                   // [len][PANEL + 1] X, then Z
  uint32_t* cand = (uint32_t*)(XT + (size_t)2 * len * (PANEL + 1));    // the candidate rows
  const bool was_done = g.done != 0;
  panel_steps<RPT>(a, g, g, a.xzs + wj, a.W, cand);
  if (!was_done) panel_post(a, g, a.po, wj, XT);
}

__global__ void __launch_bounds__(CANON_THREADS) canon_apply_kernel(const PanelArgs a) {
  extern __shared__ __align__(16) uint64_t sm[];
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;");
  panel_apply(a, *a.rec, a.po, panel_word(a.stage, a.c0, a.W / 2), blockIdx.x, gridDim.x, sm);
}

// The look-ahead schedule: per panel p two launches,
//   L1(p): CTA 0 runs panel p's pivot steps on the words a.nw (panel p's
//          word of every row as it is after panel p - 1), while CTAs 1..
//          apply panel p - 1 to the rows;
//   L2(p): CTA 0 copies panel p's pivot rows (the rows are complete through
//          panel p - 1 now) and computes its phase data, while CTAs 1..
//          compute every row's word of panel p + 1 after panel p into a.nw.
// So the serial part of a panel is the steps and the post-processing; the
// grid-wide apply runs beside the next panel's steps.  The records and pivot
// copies alternate between two buffers by panel parity (L1(p)'s apply reads
// panel p - 1's while its steps write panel p's).
template <uint32_t RPT>
__global__ void __launch_bounds__(CANON_THREADS) canon_steps_apply_kernel(const PanelArgs a) {
  extern __shared__ __align__(16) uint64_t sm[];
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;");
  if (blockIdx.x == 0) {
    if (a.steps) panel_steps<RPT>(a, *a.prev, *a.rec, a.nw, 1u, (uint32_t*)sm);
  } else if (a.wj_prev != 0xFFFFFFFFu) {
    panel_apply(a, *a.prev, a.po_prev, a.wj_prev, blockIdx.x - 1, gridDim.x - 1, sm);
  }
}

__global__ void __launch_bounds__(CANON_THREADS) canon_post_next_kernel(const PanelArgs a) {
  extern __shared__ __align__(16) uint64_t sm[];
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;");
  const uint32_t wj = panel_word(a.stage, a.c0, a.W / 2);
  if (blockIdx.x == 0) {
    panel_post(a, *a.rec, a.po, wj, sm);
  } else if (a.wj_next != 0xFFFFFFFFu) {
    panel_next(a, *a.rec, wj, a.wj_next, blockIdx.x - 1, gridDim.x - 1);
  }
}

// rows to their final positions: out[pos[r]] = row r
__global__ void canon_place_kernel(const uint64_t* xzs, const uint8_t* ph, const uint32_t* pos, uint32_t rows,
                                   uint32_t W, uint64_t* out, uint8_t* out_ph) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= rows) return;
  const uint32_t p = pos[warp];
  for (uint32_t w = lane; w < W; w += 32) out[(size_t)p * W + w] = xzs[(size_t)warp * W + w];
  if (lane == 0) out_ph[p] = ph[warp];
}

__global__ void canon_grid_init_kernel(uint32_t* pos, uint32_t rows, PanelRec* rec) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < rows) pos[r] = r;
  if (r == 0) { rec->T = 0; rec->i = 0; rec->rx = 0; rec->done = 0; }
}

// The look-ahead schedule's start: positions, both records empty, and every
// row's word of the first panel (X word 0).
__global__ void canon_look_init_kernel(uint32_t* pos, uint32_t rows, PanelRec* rec, const uint64_t* xzs,
                                       uint32_t W, uint64_t* nw) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < rows) {
    pos[r] = r;
    nw[r] = xzs[(size_t)r * W];
  }
  if (r < 2) { rec[r].T = 0; rec[r].i = 0; rec[r].rx = 0; rec[r].done = 0; }
}

struct CanonPlan {
  uint32_t cs;
  bool smem_rows;
  size_t smem_bytes;
  uint32_t RB;
};

static size_t canon_smem(uint32_t rows, uint32_t W, uint32_t RB, bool smem_rows, bool D) {
  size_t b = (size_t)(W + 1) * 8;
  if (smem_rows) b += (size_t)RB * (W + 1) * 8 * (D ? 2 : 1);
  if (D) b += (size_t)2 * W * 8;
  b += (2 + 32 + 4) * 4 + (size_t)rows * 4 + (size_t)RB * 4 + (size_t)RB * (D ? 2 : 1) + 16;
  return (b + 15) / 16 * 16;
}

static uint32_t g_canon_cs = 0;       // tuner override (0 = automatic)
static uint32_t g_canon_threads = 0;  // tuner override (0 = automatic)

static CanonPlan canon_plan(uint32_t rows, uint32_t W, bool D) {
  const size_t maxsm = (size_t)device_max_smem_optin();
  if (g_canon_cs) {
    const uint32_t cs = g_canon_cs, RB = std::max<uint32_t>(1, (rows + cs - 1) / cs);
    const bool sm = canon_smem(rows, W, RB, true, D) <= maxsm;
    return {cs, sm, canon_smem(rows, W, RB, sm, D), RB};
  }
  // measured on B200 (random full-rank stabilizers, n = 1000 / 2000 / 4000):
  // 16 CTAs beat 8 / 4 / 2 / 1 at every size (3.4 / 8.8 / 47 ms); a small
  // tableau runs in one CTA with no cluster traffic
  const uint32_t big[] = {16, 8, 4, 2, 1}, small[] = {1, 2, 4, 8, 16};
  const uint32_t* cands = rows >= 256 ? big : small;
  for (uint32_t ci = 0; ci < 5; ci++) {
    const uint32_t cs = cands[ci];
    const uint32_t RB = std::max<uint32_t>(1, (rows + cs - 1) / cs);
    if (canon_smem(rows, W, RB, true, D) <= maxsm) return {cs, true, canon_smem(rows, W, RB, true, D), RB};
  }
  const uint32_t cs = 16, RB = std::max<uint32_t>(1, (rows + cs - 1) / cs);
  return {cs, false, canon_smem(rows, W, RB, false, D), RB};
}

// One elimination launch (any mode) on a stabilizer view and, for the
// Destabilizer kinds, its destabilizer rows.  d_out receives [pivots, next i].
struct ElimSpec {
  uint64_t* xzs;
  uint8_t* ph;
  uint64_t* dxzs;
  uint8_t* dph;
  uint32_t rows, n, W;
  int phases;
  uint32_t mode, c0, i0;
  const uint32_t* d_cols;
  uint32_t ncols;
  int32_t* d_pivcols;
  int32_t* d_out;
};

static uint32_t g_canon_blocked = 0;  // 0: automatic, 1: always, 2: never

// canonicalize! by panels (canon_blocked_kernel): the cluster (16 CTAs for
// 256 rows or more, else one CTA) and whether the rows fit its shared memory.
static int launch_blocked(const ElimSpec& e, cudaStream_t st) {
  // rows per search thread (registers): 4 up to 4096 rows, else 8
  void (*kern)(const CanonArgs) = e.rows <= 4096 ? canon_blocked_kernel<4> : canon_blocked_kernel<8>;
  // the opt-in limit less the kernel's static shared memory
  cudaFuncAttributes fa{};
  QCB_CUDA(cudaFuncGetAttributes(&fa, kern));
  const size_t maxsm = (size_t)device_max_smem_optin() - fa.sharedSizeBytes;
  uint32_t cs = g_canon_cs ? g_canon_cs : (e.rows >= 256 ? 16 : 1);
  uint32_t RB = std::max<uint32_t>(1, (e.rows + cs - 1) / cs);
  bool smem_rows = blocked_layout(e.rows, e.W, RB, true).bytes <= maxsm;
  if (!smem_rows && !g_canon_cs && cs < 16) {
    cs = 16;
    RB = std::max<uint32_t>(1, (e.rows + cs - 1) / cs);
    smem_rows = blocked_layout(e.rows, e.W, RB, true).bytes <= maxsm;
  }
  const size_t bytes = blocked_layout(e.rows, e.W, RB, smem_rows).bytes;
  if (bytes > maxsm) return fail(QCB_EUNSUPPORTED, "canonicalize!: tableau too tall for the panel bookkeeping");
  CanonArgs a{};
  a.xzs = e.xzs; a.ph = e.ph; a.rows = e.rows; a.n = e.n; a.W = e.W; a.RB = RB; a.phases = e.phases;
  a.smem_rows = smem_rows ? 1 : 0;
  a.out = e.d_out;
  a.mode = ELIM_BOTH;
  if (!smem_rows) {
    QCB_CUDA(cudaMallocAsync(&a.gtmp, (size_t)e.rows * e.W * 8, st));
    QCB_CUDA(cudaMallocAsync(&a.gtmp_ph, e.rows, st));
  }
  QCB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)maxsm));
  if (cs > 8) QCB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(cs);
  cfg.blockDim = dim3(g_canon_threads ? g_canon_threads : CANON_THREADS);
  cfg.dynamicSmemBytes = bytes;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  QCB_CUDA(cudaLaunchKernelEx(&cfg, kern, a));
  QCB_LAUNCHED();
  if (!smem_rows) {
    QCB_CUDA(cudaMemcpyAsync(e.xzs, a.gtmp, (size_t)e.rows * e.W * 8, cudaMemcpyDeviceToDevice, st));
    QCB_CUDA(cudaMemcpyAsync(e.ph, a.gtmp_ph, e.rows, cudaMemcpyDeviceToDevice, st));
    QCB_CUDA(cudaFreeAsync(a.gtmp, st));
    QCB_CUDA(cudaFreeAsync(a.gtmp_ph, st));
  }
  return QCB_OK;
}

static uint32_t g_canon_grid = 0;  // 0: automatic, 1: always, 2: never (panels over the whole GPU)
static uint32_t g_canon_rpt = 0;         // tuner: rows per search thread (0: automatic; 4, 8, 16)
static uint32_t g_canon_apply_rows = 0;  // tuner: rows per apply CTA (0: automatic)
static uint32_t g_canon_pdl = 1;         // panel launches as programmatic dependents (0: plain)
static uint32_t g_canon_lookahead = 1;   // the next panel's steps beside this panel's apply (0: in turn)
// Smallest stabilizer view that runs by panels over the whole GPU (below it,
// one cluster holds the rows in shared memory).
constexpr uint32_t CANON_GRID_MIN_ROWS = 640;

// A panel launch.  With g_canon_pdl it is a programmatic dependent of the
// launch before it on the stream: its CTAs may be scheduled while that one
// finishes (each kernel waits for its predecessor with griddepcontrol.wait
// before touching memory), which hides the launch gap between the ~2 x 63
// dependent launches of each stage.
static cudaError_t launch_panel(void (*k)(const PanelArgs), uint32_t grid, uint32_t block, size_t smem,
                                cudaStream_t st, const PanelArgs& a) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = g_canon_pdl ? 1 : 0;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, a);
}

// canonicalize! by panels over the whole GPU with look-ahead
// (canon_steps_apply_kernel + canon_post_next_kernel per panel, one more
// canon_steps_apply_kernel for the last panel's apply); scratch from the
// stream-ordered pool.
static int launch_grid_lookahead(const ElimSpec& e, cudaStream_t st) {
  const uint32_t R = e.rows, W = e.W, len = W / 2;
  uint32_t* pos = nullptr;
  PanelRec* rec = nullptr;
  uint64_t *po = nullptr, *nw = nullptr, *gtmp = nullptr;
  uint8_t* gtmp_ph = nullptr;
  QCB_CUDA(cudaMallocAsync(&pos, (size_t)R * 4, st));
  QCB_CUDA(cudaMallocAsync(&rec, 2 * sizeof(PanelRec), st));
  QCB_CUDA(cudaMallocAsync(&po, (size_t)2 * PANEL * W * 8, st));
  QCB_CUDA(cudaMallocAsync(&nw, (size_t)R * 8, st));
  QCB_CUDA(cudaMallocAsync(&gtmp, (size_t)R * W * 8, st));
  QCB_CUDA(cudaMallocAsync(&gtmp_ph, R, st));
  canon_look_init_kernel<<<(R + 255) / 256, 256, 0, st>>>(pos, R, rec, e.xzs, W, nw);
  QCB_LAUNCHED();
  uint32_t rpt = g_canon_rpt ? g_canon_rpt : 4u;
  while (rpt * CANON_THREADS < R) rpt *= 2;
  void (*steps)(const PanelArgs) = rpt == 1 ? canon_steps_apply_kernel<1>
                                 : rpt == 2 ? canon_steps_apply_kernel<2>
                                 : rpt == 4 ? canon_steps_apply_kernel<4>
                                 : rpt == 8 ? canon_steps_apply_kernel<8> : canon_steps_apply_kernel<16>;
  // CTA 0 of each L1 launch runs the steps on an SM of its own (1024 threads
  // of up to 64 registers fill an SM's register file); the apply takes the
  // other SMs, one CTA each
  const uint32_t nsm = (uint32_t)device_sm_count();
  const uint32_t rows_per_cta = g_canon_apply_rows ? g_canon_apply_rows : 8u;
  const uint32_t G = std::max<uint32_t>(1, std::min<uint32_t>((R + rows_per_cta - 1) / rows_per_cta, nsm - 1));
  const uint32_t per = (R + G - 1) / G;
  const size_t l1_smem = std::max<size_t>((size_t)R * 4, (size_t)PANEL * W * 8 + (size_t)per * 9 + 16);
  const size_t l2_smem = (size_t)2 * len * (PANEL + 1) * 8;
  // the next words: a share of the rows on every other SM (the replay is a
  // serial loop over the panel's pivots per row, so the rows are spread thin)
  const uint32_t G2 = std::max<uint32_t>(1, std::min<uint32_t>(R, nsm - 1));
  QCB_CUDA(cudaFuncSetAttribute(steps, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)l1_smem));
  QCB_CUDA(cudaFuncSetAttribute(canon_post_next_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)l2_smem));
  std::vector<std::pair<uint32_t, uint32_t>> panels;  // (stage, first column)
  for (uint32_t stage = 0; stage < 2; stage++)
    for (uint32_t c0 = 0; c0 < e.n; c0 += PANEL) panels.push_back({stage, c0});
  const uint32_t P = (uint32_t)panels.size();
  PanelArgs a{};
  a.xzs = e.xzs; a.ph = e.ph; a.rows = R; a.n = e.n; a.W = W; a.phases = e.phases;
  a.pos = pos; a.out = e.d_out; a.nw = nw;
  for (uint32_t p = 0; p <= P; p++) {
    // L1(p): panel p's steps (p < P) beside panel p - 1's apply (p > 0)
    a.steps = p < P ? 1u : 0u;
    if (p < P) { a.stage = panels[p].first; a.c0 = panels[p].second; }
    a.rec = rec + (p & 1);
    a.prev = rec + ((p + 1) & 1);
    a.po_prev = po + (size_t)((p + 1) & 1) * PANEL * W;
    a.wj_prev = p > 0 ? panel_word(panels[p - 1].first, panels[p - 1].second, len) : 0xFFFFFFFFu;
    QCB_CUDA(launch_panel(steps, 1 + G, CANON_THREADS, l1_smem, st, a));
    if (p == P) break;
    // L2(p): panel p's pivot rows and phase data beside every row's next word
    a.po = po + (size_t)(p & 1) * PANEL * W;
    a.wj_next = p + 1 < P ? panel_word(panels[p + 1].first, panels[p + 1].second, len) : 0xFFFFFFFFu;
    QCB_CUDA(launch_panel(canon_post_next_kernel, 1 + G2, CANON_THREADS, l2_smem, st, a));
  }
  canon_place_kernel<<<(R * 32 + 255) / 256, 256, 0, st>>>(e.xzs, e.ph, pos, R, W, gtmp, gtmp_ph);
  QCB_LAUNCHED();
  QCB_CUDA(cudaMemcpyAsync(e.xzs, gtmp, (size_t)R * W * 8, cudaMemcpyDeviceToDevice, st));
  // without phases the reference's row swaps leave the phases in place
  if (e.phases) QCB_CUDA(cudaMemcpyAsync(e.ph, gtmp_ph, R, cudaMemcpyDeviceToDevice, st));
  QCB_CUDA(cudaFreeAsync(pos, st));
  QCB_CUDA(cudaFreeAsync(rec, st));
  QCB_CUDA(cudaFreeAsync(po, st));
  QCB_CUDA(cudaFreeAsync(nw, st));
  QCB_CUDA(cudaFreeAsync(gtmp, st));
  QCB_CUDA(cudaFreeAsync(gtmp_ph, st));
  return QCB_OK;
}

// canonicalize! by panels over the whole GPU (canon_search_kernel +
// canon_apply_kernel per panel); scratch from the stream-ordered pool.
static int launch_grid(const ElimSpec& e, cudaStream_t st) {
  if (g_canon_lookahead) return launch_grid_lookahead(e, st);
  const uint32_t R = e.rows, W = e.W, len = W / 2;
  uint32_t* pos = nullptr;
  PanelRec* rec = nullptr;
  uint64_t *po = nullptr, *gtmp = nullptr;
  uint8_t* gtmp_ph = nullptr;
  QCB_CUDA(cudaMallocAsync(&pos, (size_t)R * 4, st));
  QCB_CUDA(cudaMallocAsync(&rec, sizeof(PanelRec), st));
  QCB_CUDA(cudaMallocAsync(&po, (size_t)PANEL * W * 8, st));
  QCB_CUDA(cudaMallocAsync(&gtmp, (size_t)R * W * 8, st));
  QCB_CUDA(cudaMallocAsync(&gtmp_ph, R, st));
  canon_grid_init_kernel<<<(R + 255) / 256, 256, 0, st>>>(pos, R, rec);
  QCB_LAUNCHED();
  // rows per search thread: 4, or the fewest that fit the rows in 1024
  // threads (n = 1000: 1 / 2 / 4 / 8 rows 1.225 / 1.233 / 1.223 / 1.333 ms;
  // n = 2000: 2 / 4 / 8 rows 2.71 / 2.63 / 2.81 ms; n = 4000: 4 / 8 / 16
  // rows 7.66 / 7.86 / 11.19 ms)
  uint32_t rpt = g_canon_rpt ? g_canon_rpt : 4u;
  while (rpt * CANON_THREADS < R) rpt *= 2;
  void (*search)(const PanelArgs) = rpt == 1 ? canon_search_kernel<1>
                                  : rpt == 2 ? canon_search_kernel<2>
                                  : rpt == 4 ? canon_search_kernel<4>
                                  : rpt == 8 ? canon_search_kernel<8> : canon_search_kernel<16>;
  const size_t search_smem = (size_t)2 * len * (PANEL + 1) * 8 + (size_t)R * 4;
  // opt in always: the static shared memory counts against the default 48 KB too
  QCB_CUDA(cudaFuncSetAttribute(search, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)search_smem));
  // rows per apply CTA: 8 while that still fits one CTA per SM, else 16
  // (n = 1000: 8 / 16 rows 0.982 / 1.005 ms; n = 2000: 2.420 / 2.400 ms;
  // n = 4000: 7.89 / 7.43 ms)
  const uint32_t rows_per_cta =
      g_canon_apply_rows ? g_canon_apply_rows : (R <= 8u * (uint32_t)device_sm_count() ? 8u : 16u);
  const uint32_t G = std::max<uint32_t>(1, std::min<uint32_t>((R + rows_per_cta - 1) / rows_per_cta,
                                                              2 * (uint32_t)device_sm_count()));
  const uint32_t per = (R + G - 1) / G;
  const uint32_t threads = std::min<uint32_t>(CANON_THREADS, std::max<uint32_t>(64, 32 * per));
  const size_t apply_smem = (size_t)PANEL * W * 8 + (size_t)per * 9 + 16;
  QCB_CUDA(cudaFuncSetAttribute(canon_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)apply_smem));
  PanelArgs a{};
  a.xzs = e.xzs; a.ph = e.ph; a.rows = R; a.n = e.n; a.W = W; a.phases = e.phases;
  a.pos = pos; a.rec = rec; a.po = po; a.out = e.d_out;
  for (uint32_t stage = 0; stage < 2; stage++) {
    for (uint32_t c0 = 0; c0 < e.n; c0 += PANEL) {
      a.stage = stage;
      a.c0 = c0;
      QCB_CUDA(launch_panel(search, 1, CANON_THREADS, search_smem, st, a));
      QCB_CUDA(launch_panel(canon_apply_kernel, G, threads, apply_smem, st, a));
    }
  }
  canon_place_kernel<<<(R * 32 + 255) / 256, 256, 0, st>>>(e.xzs, e.ph, pos, R, W, gtmp, gtmp_ph);
  QCB_LAUNCHED();
  QCB_CUDA(cudaMemcpyAsync(e.xzs, gtmp, (size_t)R * W * 8, cudaMemcpyDeviceToDevice, st));
  // without phases the reference's row swaps leave the phases in place
  if (e.phases) QCB_CUDA(cudaMemcpyAsync(e.ph, gtmp_ph, R, cudaMemcpyDeviceToDevice, st));
  QCB_CUDA(cudaFreeAsync(pos, st));
  QCB_CUDA(cudaFreeAsync(rec, st));
  QCB_CUDA(cudaFreeAsync(po, st));
  QCB_CUDA(cudaFreeAsync(gtmp, st));
  QCB_CUDA(cudaFreeAsync(gtmp_ph, st));
  return QCB_OK;
}

static int eliminate(const ElimSpec& e, cudaStream_t st) {
  if (e.rows == 0) {
    const int32_t h[2] = {0, e.mode == ELIM_RREF ? -1 : (int32_t)e.i0};
    QCB_CUDA(cudaMemcpyAsync(e.d_out, h, 8, cudaMemcpyHostToDevice, st));
    QCB_CUDA(cudaStreamSynchronize(st));  // h is on this stack frame
    return QCB_OK;
  }
  const bool D = e.dxzs != nullptr;
  // by panels up to 8192 rows (the search keeps at most 8 rows per thread in registers)
  if (e.mode == ELIM_BOTH && !D && e.rows <= 8192 && g_canon_grid != 2 &&
      (g_canon_grid == 1 || e.rows >= CANON_GRID_MIN_ROWS) && g_canon_blocked != 2 && e.n > 0)
    return launch_grid(e, st);
  if (e.mode == ELIM_BOTH && !D && e.rows <= 8192 && g_canon_blocked != 2 && (g_canon_blocked == 1 || e.rows >= 64))
    return launch_blocked(e, st);
  CanonPlan p = canon_plan(e.rows, e.W, D);
  if (p.smem_bytes > (size_t)device_max_smem_optin())
    return fail(QCB_EUNSUPPORTED, "canonicalize!: tableau too tall for the cluster's bookkeeping");
  CanonArgs a{};
  a.xzs = e.xzs; a.ph = e.ph; a.dxzs = e.dxzs; a.dph = e.dph;
  a.rows = e.rows; a.n = e.n; a.W = e.W; a.RB = p.RB; a.phases = e.phases;
  a.smem_rows = p.smem_rows ? 1 : 0;
  a.out = e.d_out;
  a.mode = e.mode; a.c0 = e.c0; a.i0 = e.i0; a.cols = e.d_cols; a.ncols = e.ncols; a.pivcols = e.d_pivcols;
  const size_t nout = (size_t)e.rows * (D ? 2 : 1);
  if (!p.smem_rows) {
    QCB_CUDA(cudaMallocAsync(&a.gtmp, nout * e.W * 8, st));
    QCB_CUDA(cudaMallocAsync(&a.gtmp_ph, nout, st));
  }
  void (*kern)(const CanonArgs) =
      D ? (e.mode == ELIM_RREF ? canon_kernel<true, true> : canon_kernel<true, false>)
        : (e.mode == ELIM_RREF ? canon_kernel<false, true> : canon_kernel<false, false>);
  QCB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, device_max_smem_optin()));
  if (p.cs > 8) QCB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(p.cs);
  cfg.blockDim = dim3(g_canon_threads ? g_canon_threads : CANON_THREADS);
  cfg.dynamicSmemBytes = p.smem_bytes;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = p.cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  QCB_CUDA(cudaLaunchKernelEx(&cfg, kern, a));
  QCB_LAUNCHED();
  if (!p.smem_rows) {
    QCB_CUDA(cudaMemcpyAsync(e.xzs, a.gtmp, (size_t)e.rows * e.W * 8, cudaMemcpyDeviceToDevice, st));
    QCB_CUDA(cudaMemcpyAsync(e.ph, a.gtmp_ph, e.rows, cudaMemcpyDeviceToDevice, st));
    if (D) {
      QCB_CUDA(cudaMemcpyAsync(e.dxzs, a.gtmp + (size_t)e.rows * e.W, (size_t)e.rows * e.W * 8,
                               cudaMemcpyDeviceToDevice, st));
      QCB_CUDA(cudaMemcpyAsync(e.dph, a.gtmp_ph + e.rows, e.rows, cudaMemcpyDeviceToDevice, st));
    }
    QCB_CUDA(cudaFreeAsync(a.gtmp, st));
    QCB_CUDA(cudaFreeAsync(a.gtmp_ph, st));
  }
  return QCB_OK;
}

int canonicalize_view(uint64_t* xzs, uint8_t* ph, uint32_t rows, uint32_t n, uint32_t W, int phases,
                      int32_t* d_out, cudaStream_t st) {
  ElimSpec e{};
  e.xzs = xzs; e.ph = ph; e.rows = rows; e.n = n; e.W = W; e.phases = phases;
  e.mode = ELIM_BOTH; e.d_out = d_out;
  return eliminate(e, st);
}

// permutesystems! with a 0-based device permutation.
static int permute_dev(uint64_t* xzs, uint32_t rows, uint32_t n, uint32_t W, const uint32_t* d_perm,
                       cudaStream_t st) {
  if (!rows || !n) return QCB_OK;
  const uint32_t threads = 256, wpb = threads / 32;
  const size_t sm = (size_t)wpb * W * 8;
  if (sm > 48 * 1024) QCB_CUDA(cudaFuncSetAttribute(permute_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  const uint32_t blocks = std::min<uint32_t>((rows + wpb - 1) / wpb, 4 * (uint32_t)device_sm_count());
  permute_kernel<<<blocks, threads, sm, st>>>(xzs, rows, n, W, d_perm);
  QCB_LAUNCHED();
  return QCB_OK;
}

// The stabilizer view of a state of the given kind (src/QuantumClifford.jl
// stabilizerview): rows [off, off + rows); the Destabilizer kinds pair view
// row i with destabilizer row i.
static int state_view(const qcb_tableau* t, int kind, int32_t rank, uint32_t* off, uint32_t* rows, bool* destab) {
  *off = 0;
  *rows = t->rows;
  *destab = false;
  switch (kind) {
    case QCB_STABILIZER: return QCB_OK;
    case QCB_MIXED_STABILIZER:
      if (rank < 0 || (uint32_t)rank > t->rows) return fail(QCB_EBOUNDS, "rank out of range");
      *rows = (uint32_t)rank;
      return QCB_OK;
    case QCB_DESTABILIZER:
      if (t->rows % 2) return fail(QCB_EDIM, "destabilizer tableaux have an even number of rows");
      *off = t->rows / 2;
      *rows = t->rows / 2;
      *destab = true;
      return QCB_OK;
    case QCB_MIXED_DESTABILIZER:
      if (t->rows != 2 * t->nqubits) return fail(QCB_EDIM, "MixedDestabilizer tableaux have 2n rows");
      if (rank < 0 || (uint32_t)rank > t->nqubits) return fail(QCB_EBOUNDS, "rank out of range");
      *off = t->nqubits;
      *rows = (uint32_t)rank;
      *destab = true;
      return QCB_OK;
  }
  return fail(QCB_EARG, "bad state kind");
}

int generate_dev(uint64_t* pauli, uint8_t* pph, const uint64_t* xzs, const uint8_t* ph, uint32_t rows,
                 uint32_t W, int phases, int32_t* d_ok, int32_t* d_used, uint32_t cap, uint32_t* d_nused,
                 cudaStream_t st) {
  const size_t sm = (size_t)W * 8;
  if (sm > 48 * 1024) QCB_CUDA(cudaFuncSetAttribute(generate_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  generate_kernel<<<1, 1024, sm, st>>>(pauli, pph, xzs, ph, rows, W, phases, d_ok, d_used, cap, d_nused);
  QCB_LAUNCHED();
  return QCB_OK;
}

void set_canon_cluster(uint32_t cs) { g_canon_cs = cs; }
void set_canon_threads(uint32_t n) { g_canon_threads = n; }
void set_canon_blocked(uint32_t v) { g_canon_blocked = v; }
void set_canon_grid(uint32_t v) { g_canon_grid = v; }
void set_canon_rpt(uint32_t v) { g_canon_rpt = v; }
void set_canon_pdl(uint32_t v) { g_canon_pdl = v; }
void set_canon_lookahead(uint32_t v) { g_canon_lookahead = v; }
void set_canon_apply_rows(uint32_t v) { g_canon_apply_rows = v; }

}  // namespace qcb

using namespace qcb;

extern "C" {

int qcb_canonicalize(qcb_tableau* t, uint32_t row0, uint32_t nrows, int phases, int32_t* rx,
                     int32_t* rz, void* stream) {
  if (!t) return fail(QCB_EARG, "null tableau");
  if (row0 < 1 || (uint64_t)row0 - 1 + nrows > t->rows) return fail(QCB_EBOUNDS, "canonicalize!: row range out of bounds");
  cudaStream_t st = S(stream);
  int32_t* d_out = (int32_t*)t->scratch + 16;
  if (int s = canonicalize_view(t->xzs + (size_t)(row0 - 1) * t->W, t->phases + (row0 - 1), nrows,
                                t->nqubits, t->W, phases, d_out, st))
    return s;
  if (rx || rz) {
    int32_t h[2];
    QCB_CUDA(cudaMemcpyAsync(h, d_out, 8, cudaMemcpyDeviceToHost, st));
    QCB_CUDA(cudaStreamSynchronize(st));
    if (rx) *rx = h[0];
    if (rz) *rz = h[1];
  }
  return QCB_OK;
}

int qcb_canonicalize_state(qcb_tableau* t, int kind, int32_t rank, int phases, int32_t* rx, int32_t* rz,
                           void* stream) {
  if (!t) return fail(QCB_EARG, "null tableau");
  uint32_t off, rows;
  bool destab;
  if (int s = state_view(t, kind, rank, &off, &rows, &destab)) return s;
  cudaStream_t st = S(stream);
  ElimSpec e{};
  e.xzs = t->xzs + (size_t)off * t->W; e.ph = t->phases + off;
  if (destab) { e.dxzs = t->xzs; e.dph = t->phases; }
  e.rows = rows; e.n = t->nqubits; e.W = t->W; e.phases = phases;
  e.mode = ELIM_BOTH; e.d_out = (int32_t*)t->scratch + 16;
  if (int s = eliminate(e, st)) return s;
  if (rx || rz) {
    int32_t h[2];
    QCB_CUDA(cudaMemcpyAsync(h, e.d_out, 8, cudaMemcpyDeviceToHost, st));
    QCB_CUDA(cudaStreamSynchronize(st));
    if (rx) *rx = h[0];
    if (rz) *rz = h[1];
  }
  return QCB_OK;
}

int qcb_canonicalize_rref(qcb_tableau* t, int kind, int32_t rank, const uint32_t* cols, size_t ncols, int phases,
                          int32_t* i_out, void* stream) {
  if (!t || (ncols && !cols)) return fail(QCB_EARG, "null argument");
  uint32_t off, rows;
  bool destab;
  if (int s = state_view(t, kind, rank, &off, &rows, &destab)) return s;
  std::vector<uint32_t> c0(ncols);
  for (size_t k = 0; k < ncols; k++) {
    if (cols[k] == 0) return fail(QCB_EZEROQUBIT, "qubit indices start at 1 (NoZeroQubit)");
    if (cols[k] > t->nqubits) return fail(QCB_EBOUNDS, "canonicalize_rref!: column index exceeds the qubits");
    c0[k] = cols[k] - 1;
  }
  cudaStream_t st = S(stream);
  uint32_t* d_cols = nullptr;
  if (ncols) {
    QCB_CUDA(cudaMallocAsync(&d_cols, ncols * 4, st));
    QCB_CUDA(cudaMemcpyAsync(d_cols, c0.data(), ncols * 4, cudaMemcpyHostToDevice, st));
  }
  ElimSpec e{};
  e.xzs = t->xzs + (size_t)off * t->W; e.ph = t->phases + off;
  if (destab) { e.dxzs = t->xzs; e.dph = t->phases; }
  e.rows = rows; e.n = t->nqubits; e.W = t->W; e.phases = phases;
  e.mode = ELIM_RREF; e.d_cols = d_cols; e.ncols = (uint32_t)ncols; e.d_out = (int32_t*)t->scratch + 16;
  int s = eliminate(e, st);
  int32_t h[2] = {0, 0};
  if (s == QCB_OK) {
    if (cudaMemcpyAsync(h, e.d_out, 8, cudaMemcpyDeviceToHost, st) != cudaSuccess) s = fail(QCB_ECUDA, "copy");
  }
  if (d_cols) cudaFreeAsync(d_cols, st);
  QCB_CUDA(cudaStreamSynchronize(st));
  if (s == QCB_OK && i_out) *i_out = h[1] + 1;  // the reference's 1-based `i`
  return s;
}

int qcb_permutesystems(qcb_tableau* t, const uint32_t* perm, void* stream) {
  if (!t || !perm) return fail(QCB_EARG, "null argument");
  const uint32_t n = t->nqubits;
  std::vector<uint32_t> p0(n);
  std::vector<uint8_t> seen(n, 0);
  for (uint32_t j = 0; j < n; j++) {
    if (perm[j] < 1 || perm[j] > n || seen[perm[j] - 1]) return fail(QCB_EARG, "permutesystems!: not a permutation");
    seen[perm[j] - 1] = 1;
    p0[j] = perm[j] - 1;
  }
  cudaStream_t st = S(stream);
  if (!n || !t->rows) return QCB_OK;
  uint32_t* d_perm = nullptr;
  QCB_CUDA(cudaMallocAsync(&d_perm, (size_t)n * 4, st));
  QCB_CUDA(cudaMemcpyAsync(d_perm, p0.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st));
  int s = permute_dev(t->xzs, t->rows, n, t->W, d_perm, st);
  cudaFreeAsync(d_perm, st);
  QCB_CUDA(cudaStreamSynchronize(st));  // p0 lives on this stack frame
  return s;
}

// gott_standard_form_indices (src/canonicalization.jl:187-204) from the
// pivot columns of one stage: after the stage's elimination, row skip + a has
// its first set bit at or after column skip at the a-th pivot column, and the
// rows past the last pivot have none, so the row scan of the reference visits
// exactly the pivot columns in order.  perm is 0-based.
static void gott_perm(const std::vector<int32_t>& piv, uint32_t n, uint32_t skip, std::vector<uint32_t>& perm) {
  perm.clear();
  if (piv.empty()) {
    for (uint32_t j = 0; j < n; j++) perm.push_back(j);
    return;
  }
  std::vector<uint8_t> good(n, 0);
  for (uint32_t j = 0; j < skip; j++) perm.push_back(j);
  for (int32_t g : piv) { perm.push_back((uint32_t)g); good[g] = 1; }
  const uint32_t last = (uint32_t)piv.back();
  for (uint32_t j = skip; j <= last; j++)
    if (!good[j]) perm.push_back(j);
  for (uint32_t j = last + 1; j < n; j++) perm.push_back(j);
}

int qcb_canonicalize_gott(qcb_tableau* t, int phases, int32_t* r_out, int32_t* s_out, uint32_t* xperm,
                          uint32_t* zperm, void* stream) {
  if (!t) return fail(QCB_EARG, "null tableau");
  const uint32_t n = t->nqubits;
  cudaStream_t st = S(stream);
  int32_t* d_piv = nullptr;
  uint32_t* d_perm = nullptr;
  QCB_CUDA(cudaMallocAsync(&d_piv, (size_t)std::max<uint32_t>(n, 1) * 4, st));
  QCB_CUDA(cudaMallocAsync(&d_perm, (size_t)std::max<uint32_t>(n, 1) * 4, st));
  std::vector<int32_t> piv;
  std::vector<uint32_t> px, pz;
  int32_t h[2] = {0, 0};
  int s = QCB_OK;
  uint32_t r = 0, sz = 0;
  for (int stage = 0; stage < 2 && s == QCB_OK; stage++) {
    ElimSpec e{};
    e.xzs = t->xzs; e.ph = t->phases; e.rows = t->rows; e.n = n; e.W = t->W; e.phases = phases;
    e.mode = stage == 0 ? ELIM_X : ELIM_Z;
    e.c0 = stage == 0 ? 0 : r;
    e.i0 = stage == 0 ? 0 : r;
    e.d_pivcols = d_piv;
    e.d_out = (int32_t*)t->scratch + 16;
    if ((s = eliminate(e, st))) break;
    if (cudaMemcpyAsync(h, e.d_out, 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) { s = fail(QCB_ECUDA, "canonicalize_gott!: copy"); break; }
    const uint32_t np = (uint32_t)(t->rows ? h[0] : 0);
    piv.assign(np, 0);
    if (np && (cudaMemcpyAsync(piv.data(), d_piv, (size_t)np * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
               cudaStreamSynchronize(st) != cudaSuccess)) { s = fail(QCB_ECUDA, "canonicalize_gott!: copy"); break; }
    std::vector<uint32_t>& perm = stage == 0 ? px : pz;
    gott_perm(piv, n, stage == 0 ? 0 : r, perm);
    if (stage == 0) r = np; else sz = np;
    if (n && t->rows) {
      if (cudaMemcpyAsync(d_perm, perm.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st) != cudaSuccess) {
        s = fail(QCB_ECUDA, "canonicalize_gott!: copy");
        break;
      }
      if ((s = permute_dev(t->xzs, t->rows, n, t->W, d_perm, st))) break;
      if (cudaStreamSynchronize(st) != cudaSuccess) { s = fail(QCB_ECUDA, "canonicalize_gott!: sync"); break; }
    }
  }
  cudaFreeAsync(d_piv, st);
  cudaFreeAsync(d_perm, st);
  QCB_CUDA(cudaStreamSynchronize(st));
  if (s != QCB_OK) return s;
  if (r_out) *r_out = (int32_t)r;
  if (s_out) *s_out = (int32_t)sz;
  for (uint32_t j = 0; j < n; j++) {
    if (xperm) xperm[j] = px[j] + 1;
    if (zperm) zperm[j] = pz[j] + 1;
  }
  return QCB_OK;
}

int qcb_generate(qcb_tableau* pauli, const qcb_tableau* stab, int phases, int32_t* ok, int32_t* used_rows,
                 uint32_t cap, uint32_t* n_used, void* stream) {
  if (!pauli || !stab || !ok) return fail(QCB_EARG, "null argument");
  if (pauli->nqubits != stab->nqubits) return fail(QCB_EDIM, "generate!: sizes differ");
  cudaStream_t st = S(stream);
  int32_t* d_ok = (int32_t*)pauli->scratch + 32;
  uint32_t* d_nu = (uint32_t*)pauli->scratch + 33;
  int32_t* d_used = nullptr;
  if (used_rows && cap) QCB_CUDA(cudaMallocAsync(&d_used, (size_t)cap * 4, st));
  if (int s = generate_dev(pauli->xzs, pauli->phases, stab->xzs, stab->phases, stab->rows, stab->W, phases,
                           d_ok, d_used, used_rows ? cap : 0, d_nu, st))
    return s;
  int32_t hok = 0;
  uint32_t hnu = 0;
  QCB_CUDA(cudaMemcpyAsync(&hok, d_ok, 4, cudaMemcpyDeviceToHost, st));
  QCB_CUDA(cudaMemcpyAsync(&hnu, d_nu, 4, cudaMemcpyDeviceToHost, st));
  QCB_CUDA(cudaStreamSynchronize(st));
  if (d_used) {
    QCB_CUDA(cudaMemcpyAsync(used_rows, d_used, (size_t)std::min(hnu, cap) * 4, cudaMemcpyDeviceToHost, st));
    QCB_CUDA(cudaFreeAsync(d_used, st));
    QCB_CUDA(cudaStreamSynchronize(st));
  }
  *ok = hok;
  if (n_used) *n_used = hnu;
  return QCB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- batches of canonicalize!
// Jobs are split into classes: by 64-column panels on one CTA each (rows in
// global memory when they do not fit its shared memory), which takes the
// least SM time per job at every size measured, else by column steps on the
// smallest cluster that holds them; each class is one persistent launch on
// its own stream, forked from and joined back to the caller's stream with
// events, so the classes share the GPU.
struct CanonClass {
  uint32_t cs = 1, clusters = 1, njobs = 0;
  int blocked = 0;                 // by panels (blocked_body) or by column steps
  std::vector<void*> scratch;      // per-job row buffers of the jobs whose rows stay in global memory
  size_t smem = 0;
  qcb::CanonArgs* d_jobs = nullptr;
  uint32_t* d_head = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t done = nullptr;
};

struct qcb_canon_batch {
  std::vector<CanonClass> classes;
  int32_t* d_out = nullptr;
  uint32_t njobs = 0;
  cudaEvent_t fork = nullptr;
};

extern "C" {

int qcb_canon_batch_create(qcb_tableau* const* tabs, size_t n, int phases, uint32_t cluster, qcb_canon_batch** out) {
  using namespace qcb;
  if (!out || (n && !tabs)) return fail(QCB_EARG, "null argument");
  *out = nullptr;
  if (cluster && (cluster > 16 || (cluster & (cluster - 1)))) return fail(QCB_EARG, "cluster must be 0, 1, 2, 4, 8 or 16");
  cudaFuncAttributes fa{};
  QCB_CUDA(cudaFuncGetAttributes(&fa, canon_batch_kernel));
  const size_t maxsm = (size_t)device_max_smem_optin() - fa.sharedSizeBytes;
  // Per job: by panels on one CTA (the least SM time per job at every size
  // measured; rows in global memory when they do not fit), or the given
  // cluster; column steps for tableaux outside the panel kernel's range.
  struct Plan { uint32_t cs; int blocked; int smem_rows; size_t smem; };
  std::vector<Plan> plan(n);
  for (size_t j = 0; j < n; j++) {
    const qcb_tableau* t = tabs[j];
    if (!t) return fail(QCB_EARG, "null tableau in the batch");
    Plan& pl = plan[j];
    pl.cs = 0;
    if (t->rows >= 64 && t->rows <= 4096) {
      const uint32_t c = cluster ? cluster : 1;
      const uint32_t RB = std::max<uint32_t>(1, (t->rows + c - 1) / c);
      const size_t in_smem = blocked_layout(t->rows, t->W, RB, true).bytes;
      const size_t in_glob = blocked_layout(t->rows, t->W, RB, false).bytes;
      if (in_smem <= maxsm) pl = {c, 1, 1, in_smem};
      else if (in_glob <= maxsm) pl = {c, 1, 0, in_glob};
    }
    if (!pl.cs) {
      for (uint32_t c = 1; c <= 16; c <<= 1) {
        if (cluster && c != cluster) continue;
        const size_t sm = canon_smem(t->rows, t->W, std::max<uint32_t>(1, (t->rows + c - 1) / c), true, false);
        if (sm <= maxsm) { pl = {c, 0, 1, sm}; break; }
      }
    }
    if (!pl.cs) return fail(QCB_EUNSUPPORTED, "canonicalize! batch: a tableau does not fit the cluster's shared memory");
  }
  auto b = std::make_unique<qcb_canon_batch>();
  b->njobs = (uint32_t)n;
  QCB_CUDA(cudaMalloc(&b->d_out, std::max<size_t>(n, 1) * 8));
  QCB_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
  const uint32_t sms = (uint32_t)std::max(device_sm_count(), 1);
  for (int blk = 1; blk >= 0; blk--) {
    for (uint32_t c = 1; c <= 16; c <<= 1) {
      std::vector<uint32_t> ids;
      for (size_t j = 0; j < n; j++)
        if (plan[j].cs == c && plan[j].blocked == blk) ids.push_back((uint32_t)j);
      if (ids.empty()) continue;
      // longest first: about rows^2 * W word operations
      std::stable_sort(ids.begin(), ids.end(), [&](uint32_t x, uint32_t y) {
        return (double)tabs[x]->rows * tabs[x]->rows * tabs[x]->W > (double)tabs[y]->rows * tabs[y]->rows * tabs[y]->W;
      });
      CanonClass k;
      k.cs = c;
      k.blocked = blk;
      k.njobs = (uint32_t)ids.size();
      std::vector<CanonArgs> jobs(ids.size());
      size_t smem = 1024;
      for (size_t q = 0; q < ids.size(); q++) {
        const qcb_tableau* t = tabs[ids[q]];
        const Plan& pl = plan[ids[q]];
        CanonArgs& a = jobs[q];
        std::memset(&a, 0, sizeof(a));
        a.xzs = t->xzs; a.ph = t->phases; a.rows = t->rows; a.n = t->nqubits; a.W = t->W;
        a.RB = std::max<uint32_t>(1, (t->rows + c - 1) / c);
        a.phases = phases; a.smem_rows = pl.smem_rows; a.mode = ELIM_BOTH;
        a.out = b->d_out + 2 * ids[q];
        if (!pl.smem_rows) {
          QCB_CUDA(cudaMalloc(&a.gtmp, (size_t)t->rows * t->W * 8));
          QCB_CUDA(cudaMalloc(&a.gtmp_ph, t->rows));
          a.copy_back = 1;
          k.scratch.push_back(a.gtmp);
          k.scratch.push_back(a.gtmp_ph);
        }
        smem = std::max(smem, pl.smem);
      }
      k.smem = smem;
      // as many clusters as fit at once (one CTA per SM at this shared memory)
      k.clusters = std::max<uint32_t>(1, std::min<uint32_t>(k.njobs, sms / c));
      QCB_CUDA(cudaMalloc(&k.d_jobs, jobs.size() * sizeof(CanonArgs)));
      QCB_CUDA(cudaMalloc(&k.d_head, 4));
      QCB_CUDA(cudaMemcpy(k.d_jobs, jobs.data(), jobs.size() * sizeof(CanonArgs), cudaMemcpyHostToDevice));
      QCB_CUDA(cudaStreamCreateWithFlags(&k.st, cudaStreamNonBlocking));
      QCB_CUDA(cudaEventCreateWithFlags(&k.done, cudaEventDisableTiming));
      b->classes.push_back(k);
    }
  }
  bool big = false;
  for (auto& k : b->classes) big |= k.cs > 8;
  QCB_CUDA(cudaFuncSetAttribute(canon_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)maxsm));
  if (big) QCB_CUDA(cudaFuncSetAttribute(canon_batch_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  *out = b.release();
  return QCB_OK;
}

int qcb_canon_batch_run(qcb_canon_batch* b, void* stream) {
  using namespace qcb;
  if (!b) return fail(QCB_EARG, "null batch");
  if (!b->njobs) return QCB_OK;
  cudaStream_t st = S(stream);
  QCB_CUDA(cudaEventRecord(b->fork, st));
  for (auto& k : b->classes) {
    QCB_CUDA(cudaStreamWaitEvent(k.st, b->fork, 0));
    QCB_CUDA(cudaMemsetAsync(k.d_head, 0, 4, k.st));
    CanonBatchArgs a{k.d_jobs, k.njobs, k.d_head, k.blocked};
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(k.clusters * k.cs);
    cfg.blockDim = dim3(CANON_THREADS);
    cfg.dynamicSmemBytes = k.smem;
    cfg.stream = k.st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = k.cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    QCB_CUDA(cudaLaunchKernelEx(&cfg, canon_batch_kernel, a));
    QCB_LAUNCHED();
    QCB_CUDA(cudaEventRecord(k.done, k.st));
    QCB_CUDA(cudaStreamWaitEvent(st, k.done, 0));
  }
  return QCB_OK;
}

int qcb_canon_batch_ranks(const qcb_canon_batch* b, int32_t* rx, int32_t* rz) {
  using namespace qcb;
  if (!b) return fail(QCB_EARG, "null batch");
  std::vector<int32_t> h((size_t)b->njobs * 2);
  QCB_CUDA(cudaDeviceSynchronize());
  if (b->njobs) QCB_CUDA(cudaMemcpy(h.data(), b->d_out, h.size() * 4, cudaMemcpyDeviceToHost));
  for (uint32_t j = 0; j < b->njobs; j++) {
    if (rx) rx[j] = h[2 * j];
    if (rz) rz[j] = h[2 * j + 1];
  }
  return QCB_OK;
}

int qcb_canon_batch_destroy(qcb_canon_batch* b) {
  if (!b) return QCB_OK;
  for (auto& k : b->classes) {
    for (void* p : k.scratch) cudaFree(p);
    cudaFree(k.d_jobs);
    cudaFree(k.d_head);
    if (k.st) cudaStreamDestroy(k.st);
    if (k.done) cudaEventDestroy(k.done);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  cudaFree(b->d_out);
  delete b;
  return QCB_OK;
}

}  // extern "C"
