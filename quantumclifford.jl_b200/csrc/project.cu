// project.cu -- project! for Stabilizer, MixedStabilizer, Destabilizer and
// MixedDestabilizer tableaux (src/project_trace_reset.jl:231-439).
//
// One thread-block cluster projects a list of Paulis in order on one state.
// The tableau stays in global memory (it is L2 resident at these sizes).  Per
// Pauli:
//   1. every CTA computes comm(pauli, row) for its share of the rows (warp per
//      row, parity of popcounts) into a flag array, and the first
//      anticommuting row of each range the reference scans;
//   2. after a cluster barrier every CTA reads all CTAs' minima through
//      distributed shared memory, so all take the same branch;
//   3. the row swaps of the MixedDestabilizer logical branch are done by CTA 0
//      (flags swapped with the rows), then every CTA left-multiplies its
//      anticommuting rows by the pivot row exactly as anticomm_update_rows
//      (:319-335) does (comm is evaluated on the rows before any update, and
//      the pivot row is never updated, so the row updates are independent);
//   4. CTA 0 does the row copies, rank update and the result.
// The commuting branch of Stabilizer / MixedStabilizer needs canonicalize! +
// generate!; the kernel stops there and the host runs those kernels before
// resuming with the next Pauli.
#include <cooperative_groups.h>

#include <algorithm>

#include "qcb_internal.h"

namespace cg = cooperative_groups;

namespace qcb {

int canonicalize_view(uint64_t* xzs, uint8_t* ph, uint32_t rows, uint32_t n, uint32_t W, int phases,
                      int32_t* d_out, cudaStream_t st);
int generate_dev(uint64_t* pauli, uint8_t* pph, const uint64_t* xzs, const uint8_t* ph, uint32_t rows,
                 uint32_t W, int phases, int32_t* d_ok, int32_t* d_used, uint32_t cap, uint32_t* d_nused,
                 cudaStream_t st);

__device__ __forceinline__ void mul_step_p(uint64_t x1, uint64_t z1, uint64_t& x2, uint64_t& z2,
                                           uint64_t& c1, uint64_t& c2) {
  const uint64_t nx = x1 ^ x2, nz = z1 ^ z2;
  const uint64_t x1z2 = x1 & z2;
  const uint64_t anti = (x2 & z1) ^ x1z2;
  c2 ^= (c1 ^ nx ^ nz ^ x1z2) & anti;
  c1 ^= anti;
  x2 = nx;
  z2 = nz;
}

enum : int32_t { PST_OK = 0, PST_NEED_CANON = 1, PST_BADSTRUCT = 2 };

struct ProjArgs {
  uint64_t* xzs;
  uint8_t* ph;
  uint32_t rows, n, W;
  int kind;
  int32_t* rank;         // device rank (mixed kinds)
  const uint64_t* paulis;
  const uint8_t* pph;
  uint32_t j0, k;        // project Paulis [j0, k)
  int keep_result, phases;
  int32_t* anticom;
  int32_t* result;
  int32_t* status;       // [0] = status, [1] = index reached
  uint8_t* flags;        // rows
  const uint32_t* qubits;  // projectX!/Y!/Z!: Pauli j is the single-qubit Pauli on qubits[j] (0-based), or null
  uint32_t basis;          // with qubits: bit 0 = X component, bit 1 = Z component
  const uint8_t* rand_ph;  // projectrand!: phase (0 or 2) given to the new stabilizer row of Pauli j, or null
};

constexpr uint32_t PROJ_THREADS = 1024;

// row m <- row i * row m (mul_left!(tab, m, i)), warp-cooperative.
__device__ __forceinline__ void warp_rowmul(uint64_t* xzs, uint8_t* ph, uint32_t W, uint32_t m,
                                            const uint64_t* piv, uint32_t pph, bool phases,
                                            uint32_t lane) {
  const uint32_t len = W / 2;
  uint64_t* row = xzs + (size_t)m * W;
  uint64_t c1 = 0, c2 = 0;
  for (uint32_t w = lane; w < len; w += 32) {
    uint64_t x2 = row[w], z2 = row[len + w];
    mul_step_p(piv[w], piv[len + w], x2, z2, c1, c2);
    row[w] = x2;
    row[len + w] = z2;
  }
  if (phases) {
    const uint32_t s =
        __reduce_add_sync(0xFFFFFFFFu, (uint32_t)(__popcll(c1) + 2 * __popcll(c2)) & 3u) & 3u;
    if (lane == 0) ph[m] = (uint8_t)((s + ph[m] + pph) & 3u);
  }
}

__global__ void __launch_bounds__(PROJ_THREADS) project_kernel(const ProjArgs a) {
  cg::cluster_group cl = cg::this_cluster();
  const uint32_t me = cl.block_rank(), CS = cl.num_blocks();
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const uint32_t gw = me * nwarps + warp, NW = CS * nwarps;
  const uint32_t W = a.W, len = W / 2;
  extern __shared__ __align__(16) uint64_t smem[];
  uint64_t* P = smem;            // W words: the Pauli
  uint64_t* piv = smem + W;      // W words: the pivot row
  __shared__ uint32_t mins[3];   // first anticommuting: stab range, logical X, logical Z
  __shared__ int32_t dec[8];     // decision broadcast

  const uint32_t rows = a.rows;
  for (uint32_t j = a.j0; j < a.k; j++) {
    const bool single = a.qubits != nullptr;
    uint32_t wq = 0;
    uint64_t bq = 0;
    if (single) {
      wq = a.qubits[j] >> 6;
      bq = 1ull << (a.qubits[j] & 63);
      for (uint32_t w = tid; w < W; w += blockDim.x)
        P[w] = (((a.basis & 1u) && w == wq) ? bq : 0ull) | (((a.basis & 2u) && w == len + wq) ? bq : 0ull);
    } else {
      const uint64_t* pj = a.paulis + (size_t)j * W;
      for (uint32_t w = tid; w < W; w += blockDim.x) P[w] = pj[w];
    }
    if (tid < 3) mins[tid] = 0xFFFFFFFFu;
    const uint32_t pphase = single ? 0u : a.pph[j];
    int32_t r = a.kind == QCB_STABILIZER ? (int32_t)rows : (a.kind == QCB_DESTABILIZER ? (int32_t)(rows / 2) : *a.rank);
    __syncthreads();
    const uint32_t nn = (a.kind == QCB_DESTABILIZER || a.kind == QCB_MIXED_DESTABILIZER) ? rows / 2 : rows;
    // 1. comm flags for every row and the first anticommuting rows
    auto note = [&](uint32_t m, uint32_t c) {
      a.flags[m] = (uint8_t)c;
      if (c) {
        if (a.kind == QCB_STABILIZER || a.kind == QCB_MIXED_STABILIZER) {
          if (m < (uint32_t)r) atomicMin(&mins[0], m);
        } else {
          if (m >= nn && m < nn + (uint32_t)r) atomicMin(&mins[0], m - nn);
          if (a.kind == QCB_MIXED_DESTABILIZER) {
            if (m >= (uint32_t)r && m < nn) atomicMin(&mins[1], m);
            if (m >= nn + (uint32_t)r) atomicMin(&mins[2], m);
          }
        }
      }
    };
    if (single) {
      // comm with a single-qubit Pauli is one bit of the row (the isX / isZ /
      // isXorZ tests of project_cond!, src/project_trace_reset.jl:476-479)
      for (uint32_t m = me * blockDim.x + tid; m < rows; m += CS * blockDim.x) {
        const uint64_t* row = a.xzs + (size_t)m * W;
        uint32_t c = 0;
        if (a.basis & 1u) c ^= (uint32_t)((row[len + wq] & bq) != 0);
        if (a.basis & 2u) c ^= (uint32_t)((row[wq] & bq) != 0);
        note(m, c);
      }
    } else {
      for (uint32_t m = gw; m < rows; m += NW) {
        const uint64_t* row = a.xzs + (size_t)m * W;
        uint64_t acc = 0;
        for (uint32_t w = lane; w < len; w += 32) acc ^= (P[len + w] & row[w]) ^ (P[w] & row[len + w]);
        const uint32_t c = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)__popcll(acc)) & 1u;
        if (lane == 0) note(m, c);
      }
    }
    __syncthreads();
    cl.sync();
    // 2. uniform decision
    if (tid == 0) {
      uint32_t m0 = 0xFFFFFFFFu, m1 = 0xFFFFFFFFu, m2 = 0xFFFFFFFFu;
      for (uint32_t q = 0; q < CS; q++) {
        uint32_t* rm = cl.map_shared_rank(mins, q);
        m0 = min(m0, rm[0]); m1 = min(m1, rm[1]); m2 = min(m2, rm[2]);
      }
      // dec: [0] branch, [1] pivot row, [2] anticom (1-based), [3] update r, [4] update anticommutes
      int32_t branch = 0, pivrow = -1, anticom = 0;
      if (m0 != 0xFFFFFFFFu) {
        branch = 1;  // anticommutes with a stabilizer row
        anticom = (int32_t)m0 + 1;
      } else if (a.kind == QCB_MIXED_DESTABILIZER && (m1 != 0xFFFFFFFFu || m2 != 0xFFFFFFFFu)) {
        branch = 2;  // anticommutes with a logical operator
        anticom = (int32_t)(m1 != 0xFFFFFFFFu ? m1 : m2) + 1;  // 1-based anticomlog
      } else {
        branch = 0;
      }
      if (branch == 1) {
        pivrow = (a.kind == QCB_STABILIZER || a.kind == QCB_MIXED_STABILIZER) ? anticom - 1 : (int32_t)nn + anticom - 1;
      } else if (branch == 2) {
        pivrow = (int32_t)nn + r;  // row n+r+1 (1-based) after the swaps
      }
      dec[0] = branch; dec[1] = pivrow; dec[2] = anticom;
    }
    __syncthreads();
    const int32_t branch = dec[0];
    if (branch == 0) {
      // commutes with every stabilizer row
      bool stop = false;
      if (a.kind == QCB_STABILIZER || a.kind == QCB_MIXED_STABILIZER) {
        if (a.keep_result || a.kind == QCB_MIXED_STABILIZER) stop = true;
        else if (me == 0 && tid == 0) { a.anticom[j] = 0; a.result[j] = -1; }
      } else if (a.kind == QCB_DESTABILIZER && nn != a.n) {
        if (me == 0 && tid == 0) { a.status[0] = PST_BADSTRUCT; a.status[1] = (int32_t)j; }
        cl.sync();
        return;
      } else if (me == 0 && warp == 0) {
        int32_t res = -1;
        if (a.keep_result) {
          // new_pauli = product of the stabilizer rows whose destabilizer
          // anticommutes with the Pauli, phase starting from the Pauli's
          uint64_t c1 = 0, c2 = 0;
          uint32_t extra = pphase;
          uint64_t* buf = piv;  // the pivot buffer is free in this branch
          for (uint32_t w = lane; w < W; w += 32) buf[w] = 0;
          __syncwarp();
          for (uint32_t i = 0; i < (uint32_t)r; i++) {
            if (!a.flags[i]) continue;  // comm(pauli, destabilizer row i)
            const uint64_t* srow = a.xzs + (size_t)(nn + i) * W;
            for (uint32_t w = lane; w < len; w += 32) {
              uint64_t x2 = buf[w], z2 = buf[len + w];
              mul_step_p(srow[w], srow[len + w], x2, z2, c1, c2);
              buf[w] = x2;
              buf[len + w] = z2;
            }
            __syncwarp();
            extra += a.ph[nn + i];
          }
          const uint32_t s =
              __reduce_add_sync(0xFFFFFFFFu, (uint32_t)(__popcll(c1) + 2 * __popcll(c2)) & 3u) & 3u;
          res = a.phases ? (int32_t)((s + extra) & 3u) : (int32_t)(pphase & 3u);
        }
        if (lane == 0) { a.anticom[j] = 0; a.result[j] = res; }
      }
      if (stop) {
        if (me == 0 && tid == 0) { a.status[0] = PST_NEED_CANON; a.status[1] = (int32_t)j; }
        cl.sync();
        return;
      }
      cl.sync();
      continue;
    }
    // 3. swaps (MixedDestabilizer logical branch), done by CTA 0
    if (branch == 2) {
      if (me == 0) {
        const uint32_t al = (uint32_t)dec[2];  // 1-based anticomlog
        auto swaprow = [&](uint32_t u, uint32_t v) {  // 0-based
          if (u == v) return;
          uint64_t* ru = a.xzs + (size_t)u * W;
          uint64_t* rv = a.xzs + (size_t)v * W;
          for (uint32_t w = tid; w < W; w += blockDim.x) { uint64_t t = ru[w]; ru[w] = rv[w]; rv[w] = t; }
          if (tid == 0) {
            uint8_t t = a.ph[u]; a.ph[u] = a.ph[v]; a.ph[v] = t;
            uint8_t f = a.flags[u]; a.flags[u] = a.flags[v]; a.flags[v] = f;
          }
          __syncthreads();
        };
        const uint32_t ru = (uint32_t)r;
        if (al <= nn) {
          swaprow(ru + nn, al - 1);
          if (nn != ru + 1 && al != ru + 1) swaprow(ru, al + nn - 1);
        } else {
          swaprow(ru, al - nn - 1);
          swaprow(ru + nn, al - 1);
        }
      }
      cl.sync();
    }
    // 4. row updates (anticomm_update_rows or the Stabilizer loop)
    const uint32_t pivrow = (uint32_t)dec[1];
    for (uint32_t w = tid; w < W; w += blockDim.x) piv[w] = a.xzs[(size_t)pivrow * W + w];
    __syncthreads();
    const uint32_t pph = a.ph[pivrow];
    if (a.kind == QCB_STABILIZER || a.kind == QCB_MIXED_STABILIZER) {
      const uint32_t ac = (uint32_t)dec[2];
      for (uint32_t m = ac + gw; m < (uint32_t)r; m += NW)
        if (a.flags[m]) warp_rowmul(a.xzs, a.ph, W, m, piv, pph, a.phases != 0, lane);
    } else {
      const uint32_t ru = branch == 2 ? (uint32_t)r + 1 : (uint32_t)r;
      const uint32_t ac = branch == 2 ? (uint32_t)r + 1 : (uint32_t)dec[2];
      for (uint32_t m = gw; m < 2 * nn; m += NW) {
        if (!a.flags[m] || m == pivrow) continue;
        if (m >= ru && m < nn) warp_rowmul(a.xzs, a.ph, W, m, piv, pph, a.phases != 0, lane);
        else if (m >= nn + ac && m < 2 * nn) warp_rowmul(a.xzs, a.ph, W, m, piv, pph, a.phases != 0, lane);
        else if (m < ru && m != ac - 1) warp_rowmul(a.xzs, a.ph, W, m, piv, pph, false, lane);
      }
    }
    cl.sync();
    // 5. row copies, rank, outputs (CTA 0)
    if (me == 0) {
      if (a.kind == QCB_STABILIZER || a.kind == QCB_MIXED_STABILIZER) {
        const uint32_t ac = (uint32_t)dec[2];
        for (uint32_t w = tid; w < W; w += blockDim.x) a.xzs[(size_t)(ac - 1) * W + w] = P[w];
        if (tid == 0) {
          // projectrand!: the undetermined outcome gets a random sign
          const int32_t rp = a.rand_ph ? (int32_t)a.rand_ph[j] : -1;
          a.ph[ac - 1] = (uint8_t)(rp >= 0 ? rp : (int32_t)pphase);
          a.anticom[j] = (int32_t)ac;
          a.result[j] = rp;
        }
      } else {
        const uint32_t ac = branch == 2 ? (uint32_t)r + 1 : (uint32_t)dec[2];
        // destabilizer[ac] = stabilizer[ac]; stabilizer[ac] = pauli
        for (uint32_t w = tid; w < W; w += blockDim.x) {
          a.xzs[(size_t)(ac - 1) * W + w] = a.xzs[(size_t)(nn + ac - 1) * W + w];
        }
        __syncthreads();
        for (uint32_t w = tid; w < W; w += blockDim.x) a.xzs[(size_t)(nn + ac - 1) * W + w] = P[w];
        if (tid == 0) {
          const int32_t rp = a.rand_ph ? (int32_t)a.rand_ph[j] : -1;
          a.ph[ac - 1] = a.ph[nn + ac - 1];
          a.ph[nn + ac - 1] = (uint8_t)(rp >= 0 ? rp : (int32_t)pphase);
          if (branch == 2) *a.rank = r + 1;
          a.anticom[j] = (int32_t)(branch == 2 ? r + 1 : (int32_t)ac);
          a.result[j] = rp;
        }
      }
    }
    cl.sync();
  }
  if (me == 0 && tid == 0) { a.status[0] = PST_OK; a.status[1] = (int32_t)a.k; }
}

// ---------------------------------------------------------------------------
// project_smem_kernel: the same projections with the whole tableau held in
// the cluster's shared memory (CTA c owns rows [c*RB, c*RB + RB), row stride
// W+1 words).  Per Pauli there are two cluster barriers: one after every CTA
// has published the first anticommuting row of each range it owns (every CTA
// then reads all of them through distributed shared memory and takes the
// same decision), one after every CTA has fetched the pivot row.  The row
// products then run on local rows only, and the row copies are done by the
// rows' owners from their local copies of the pivot and the Pauli (neither
// row is among the updated ones).  Rows are read from and written back to
// global memory once per launch.
struct ProjSmemArgs {
  ProjArgs a;
  uint32_t RB;
};

// Lanes per row: the smallest power of two >= the words of one half, at most 32.
__device__ __forceinline__ uint32_t group_lanes(uint32_t len) {
  uint32_t g = 1;
  while (g < len && g < 32) g <<= 1;
  return g;
}

__global__ void __launch_bounds__(PROJ_THREADS) project_smem_kernel(const ProjSmemArgs pa) {
  const ProjArgs& a = pa.a;
  cg::cluster_group cl = cg::this_cluster();
  const uint32_t me = cl.block_rank(), CS = cl.num_blocks();
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const uint32_t W = a.W, len = W / 2, WS = W + 1, RB = pa.RB;
  const uint32_t rows = a.rows;
  const uint32_t r0 = me * RB;
  const uint32_t nloc = r0 < rows ? min(RB, rows - r0) : 0u;
  const uint32_t G = group_lanes(len), GPW = 32 / G;  // lanes per row, rows per warp pass
  const uint32_t gl = lane % G, gi = lane / G;

  extern __shared__ __align__(16) uint64_t smem[];
  uint64_t* P = smem;                       // W: the Pauli
  uint64_t* piv = P + W;                    // W: the pivot row / partial product
  uint64_t* R = piv + W + 1;                // RB * WS: the rows
  uint8_t* ph = (uint8_t*)(R + (size_t)RB * WS);  // RB
  uint8_t* fl = ph + RB;                    // RB: comm flags
  uint32_t* slot = (uint32_t*)(((uintptr_t)(fl + RB) + 15) & ~(uintptr_t)15);  // [2][4]
  uint32_t* mins = slot + 8;                // 3
  int32_t* dec = (int32_t*)(mins + 4);      // 8

  auto ROW = [&](uint32_t lr) -> uint64_t* { return R + (size_t)lr * WS; };
  // (owner CTA, local row) of a global row
  auto owner_of = [&](uint32_t m) -> uint32_t { return m / RB; };

  for (uint32_t lr = warp; lr < nloc; lr += nwarps)
    for (uint32_t w = lane; w < W; w += 32) ROW(lr)[w] = a.xzs[(size_t)(r0 + lr) * W + w];
  for (uint32_t lr = tid; lr < nloc; lr += blockDim.x) ph[lr] = a.ph[r0 + lr];
  const bool destab = a.kind == QCB_DESTABILIZER || a.kind == QCB_MIXED_DESTABILIZER;
  const uint32_t nn = destab ? rows / 2 : rows;
  int32_t r = a.kind == QCB_STABILIZER ? (int32_t)rows : (a.kind == QCB_DESTABILIZER ? (int32_t)(rows / 2) : *a.rank);
  __syncthreads();
  cl.sync();

  uint32_t status = PST_OK, jstop = a.k;
  for (uint32_t j = a.j0; j < a.k; j++) {
    const uint32_t par = j & 1;
    const bool single = a.qubits != nullptr;
    uint32_t wq = 0;
    uint64_t bq = 0;
    if (single) {
      wq = a.qubits[j] >> 6;
      bq = 1ull << (a.qubits[j] & 63);
      for (uint32_t w = tid; w < W; w += blockDim.x)
        P[w] = (((a.basis & 1u) && w == wq) ? bq : 0ull) | (((a.basis & 2u) && w == len + wq) ? bq : 0ull);
    } else {
      const uint64_t* pj = a.paulis + (size_t)j * W;
      for (uint32_t w = tid; w < W; w += blockDim.x) P[w] = pj[w];
    }
    if (tid < 3) mins[tid] = 0xFFFFFFFFu;
    const uint32_t pphase = single ? 0u : a.pph[j];
    __syncthreads();
    // 1. comm flags of the local rows and the first anticommuting row of each range
    auto note = [&](uint32_t m, uint32_t c) {
      if (!c) return;
      if (!destab) {
        if (m < (uint32_t)r) atomicMin(&mins[0], m);
      } else {
        if (m >= nn && m < nn + (uint32_t)r) atomicMin(&mins[0], m - nn);
        if (a.kind == QCB_MIXED_DESTABILIZER) {
          if (m >= (uint32_t)r && m < nn) atomicMin(&mins[1], m);
          if (m >= nn + (uint32_t)r) atomicMin(&mins[2], m);
        }
      }
    };
    if (single) {
      for (uint32_t lr = tid; lr < nloc; lr += blockDim.x) {
        const uint64_t* row = ROW(lr);
        uint32_t c = 0;
        if (a.basis & 1u) c ^= (uint32_t)((row[len + wq] & bq) != 0);
        if (a.basis & 2u) c ^= (uint32_t)((row[wq] & bq) != 0);
        fl[lr] = (uint8_t)c;
        note(r0 + lr, c);
      }
    } else {
      for (uint32_t base = warp * GPW; base < nloc; base += nwarps * GPW) {
        const uint32_t lr = base + gi;
        uint64_t acc = 0;
        if (lr < nloc) {
          const uint64_t* row = ROW(lr);
          for (uint32_t w = gl; w < len; w += G) acc ^= (P[len + w] & row[w]) ^ (P[w] & row[len + w]);
        }
        uint32_t c = (uint32_t)__popcll(acc);
        for (uint32_t off = G >> 1; off; off >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, off);
        c &= 1u;
        if (gl == 0 && lr < nloc) {
          fl[lr] = (uint8_t)c;
          note(r0 + lr, c);
        }
      }
    }
    __syncthreads();
    if (tid < 3) slot[par * 4 + tid] = mins[tid];
    cl.sync();
    // 2. the same decision in every CTA
    if (warp == 0) {
      uint32_t m0 = 0xFFFFFFFFu, m1 = 0xFFFFFFFFu, m2 = 0xFFFFFFFFu;
      if (lane < CS) {
        const uint32_t* rs = cl.map_shared_rank(slot + par * 4, lane);
        m0 = rs[0]; m1 = rs[1]; m2 = rs[2];
      }
      m0 = __reduce_min_sync(0xFFFFFFFFu, m0);
      m1 = __reduce_min_sync(0xFFFFFFFFu, m1);
      m2 = __reduce_min_sync(0xFFFFFFFFu, m2);
      if (lane == 0) {
        int32_t branch = 0, pivrow = -1, anticom = 0;
        if (m0 != 0xFFFFFFFFu) {
          branch = 1;
          anticom = (int32_t)m0 + 1;
          pivrow = destab ? (int32_t)nn + anticom - 1 : anticom - 1;
        } else if (a.kind == QCB_MIXED_DESTABILIZER && (m1 != 0xFFFFFFFFu || m2 != 0xFFFFFFFFu)) {
          branch = 2;
          anticom = (int32_t)(m1 != 0xFFFFFFFFu ? m1 : m2) + 1;  // 1-based anticomlog
          pivrow = (int32_t)nn + r;
        }
        dec[0] = branch; dec[1] = pivrow; dec[2] = anticom;
      }
    }
    __syncthreads();
    const int32_t branch = dec[0];
    if (branch == 0) {
      if (!destab) {
        if (a.keep_result || a.kind == QCB_MIXED_STABILIZER) { status = PST_NEED_CANON; jstop = j; break; }
        if (me == 0 && tid == 0) { a.anticom[j] = 0; a.result[j] = -1; }
        continue;
      }
      if (a.kind == QCB_DESTABILIZER && nn != a.n) { status = PST_BADSTRUCT; jstop = j; break; }
      if (!a.keep_result) {
        if (me == 0 && tid == 0) { a.anticom[j] = 0; a.result[j] = -1; }
        continue;
      }
      // result: the product of the stabilizer rows i < r whose destabilizer
      // row anticommutes with the Pauli (the stabilizer rows commute, so the
      // per-CTA partial products can be combined in any order with the exact
      // phase).  Warp 0 of each CTA multiplies its own stabilizer rows.
      if (warp == 0) {
        uint64_t c1 = 0, c2 = 0;
        uint32_t extra = 0;
        for (uint32_t w = lane; w < W; w += 32) piv[w] = 0;
        __syncwarp();
        for (uint32_t lr = 0; lr < nloc; lr++) {
          const uint32_t m = r0 + lr;
          if (m < nn || m >= nn + (uint32_t)r) continue;
          const uint32_t i = m - nn;  // destabilizer partner row i
          const uint32_t o = owner_of(i);
          const uint8_t f = o == me ? fl[i - r0] : *cl.map_shared_rank(fl + (i - o * RB), o);
          if (!f) continue;
          const uint64_t* srow = ROW(lr);
          for (uint32_t w = lane; w < len; w += 32) {
            uint64_t x2 = piv[w], z2 = piv[len + w];
            mul_step_p(srow[w], srow[len + w], x2, z2, c1, c2);
            piv[w] = x2;
            piv[len + w] = z2;
          }
          __syncwarp();
          extra += ph[lr];
        }
        const uint32_t s = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)(__popcll(c1) + 2 * __popcll(c2)) & 3u) & 3u;
        if (lane == 0) piv[W] = (uint64_t)((s + extra) & 3u);
      }
      cl.sync();
      if (me == 0 && warp == 0) {
        // combine the CTAs' partial products in CTA order into P's buffer
        uint64_t c1 = 0, c2 = 0;
        uint32_t extra = pphase;
        for (uint32_t w = lane; w < W; w += 32) P[w] = 0;
        __syncwarp();
        for (uint32_t q = 0; q < CS; q++) {
          const uint64_t* pq = q == 0 ? piv : cl.map_shared_rank(piv, q);
          for (uint32_t w = lane; w < len; w += 32) {
            uint64_t x2 = P[w], z2 = P[len + w];
            mul_step_p(pq[w], pq[len + w], x2, z2, c1, c2);
            P[w] = x2;
            P[len + w] = z2;
          }
          __syncwarp();
          extra += (uint32_t)pq[W];
        }
        const uint32_t s = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)(__popcll(c1) + 2 * __popcll(c2)) & 3u) & 3u;
        if (lane == 0) {
          a.anticom[j] = 0;
          a.result[j] = a.phases ? (int32_t)((s + extra) & 3u) : (int32_t)(pphase & 3u);
        }
      }
      continue;
    }
    // 3. MixedDestabilizer logical branch: the row swaps (rare), by CTA 0
    //    through distributed shared memory
    if (branch == 2) {
      if (me == 0) {
        const uint32_t al = (uint32_t)dec[2];
        auto swaprow = [&](uint32_t u, uint32_t v) {
          if (u == v) return;
          const uint32_t ou = owner_of(u), ov = owner_of(v);
          uint64_t* ru = cl.map_shared_rank(R + (size_t)(u - ou * RB) * WS, ou);
          uint64_t* rv = cl.map_shared_rank(R + (size_t)(v - ov * RB) * WS, ov);
          for (uint32_t w = tid; w < W; w += blockDim.x) { const uint64_t t = ru[w]; ru[w] = rv[w]; rv[w] = t; }
          if (tid == 0) {
            uint8_t* pu = cl.map_shared_rank(ph + (u - ou * RB), ou);
            uint8_t* pv = cl.map_shared_rank(ph + (v - ov * RB), ov);
            uint8_t t = *pu; *pu = *pv; *pv = t;
            uint8_t* fu = cl.map_shared_rank(fl + (u - ou * RB), ou);
            uint8_t* fv = cl.map_shared_rank(fl + (v - ov * RB), ov);
            t = *fu; *fu = *fv; *fv = t;
          }
          __syncthreads();
        };
        const uint32_t ru = (uint32_t)r;
        if (al <= nn) {
          swaprow(ru + nn, al - 1);
          if (nn != ru + 1 && al != ru + 1) swaprow(ru, al + nn - 1);
        } else {
          swaprow(ru, al - nn - 1);
          swaprow(ru + nn, al - 1);
        }
      }
      cl.sync();
    }
    // 4. every CTA fetches the pivot row, then a barrier before its owner may
    //    overwrite it
    const uint32_t pivrow = (uint32_t)dec[1];
    {
      const uint32_t o = owner_of(pivrow), lr = pivrow - o * RB;
      const uint64_t* src = o == me ? ROW(lr) : cl.map_shared_rank(R + (size_t)lr * WS, o);
      for (uint32_t w = tid; w < W; w += blockDim.x) piv[w] = src[w];
      if (tid == 0) piv[W] = o == me ? ph[lr] : *cl.map_shared_rank(ph + lr, o);
    }
    cl.sync();
    const uint32_t pph = (uint32_t)piv[W];
    // 5. row products on local rows (anticomm_update_rows or the Stabilizer loop)
    const uint32_t ac = branch == 2 ? (uint32_t)r + 1 : (uint32_t)dec[2];
    const uint32_t ru = branch == 2 ? (uint32_t)r + 1 : (uint32_t)r;
    for (uint32_t base = warp * GPW; base < nloc; base += nwarps * GPW) {
      const uint32_t lr = base + gi;
      const uint32_t m = r0 + lr;
      int mode = 0;  // 0: skip, 1: with phase, 2: without phase
      if (lr < nloc && fl[lr] && m != pivrow) {
        if (!destab) mode = (m >= ac && m < (uint32_t)r) ? 1 : 0;
        else if (m >= ru && m < nn) mode = 1;
        else if (m >= nn + ac && m < 2 * nn) mode = 1;
        else if (m < ru && m != ac - 1) mode = 2;
      }
      uint64_t c1 = 0, c2 = 0;
      if (mode) {
        uint64_t* row = ROW(lr);
        for (uint32_t w = gl; w < len; w += G) {
          uint64_t x2 = row[w], z2 = row[len + w];
          mul_step_p(piv[w], piv[len + w], x2, z2, c1, c2);
          row[w] = x2;
          row[len + w] = z2;
        }
      }
      uint32_t sc = (uint32_t)(__popcll(c1) + 2 * __popcll(c2));
      for (uint32_t off = G >> 1; off; off >>= 1) sc += __shfl_xor_sync(0xFFFFFFFFu, sc, off);
      if (gl == 0 && mode == 1 && a.phases) ph[lr] = (uint8_t)((sc + ph[lr] + pph) & 3u);
    }
    // 6. row copies by the owners, outputs by CTA 0
    const int32_t rp = a.rand_ph ? (int32_t)a.rand_ph[j] : -1;
    if (!destab) {
      const uint32_t dst = ac - 1;
      if (owner_of(dst) == me) {
        const uint32_t lr = dst - r0;
        for (uint32_t w = tid; w < W; w += blockDim.x) ROW(lr)[w] = P[w];
        if (tid == 0) ph[lr] = (uint8_t)(rp >= 0 ? rp : (int32_t)pphase);
      }
    } else {
      // destabilizer[ac] = stabilizer[ac] (the pivot row); stabilizer[ac] = pauli
      const uint32_t dd = ac - 1, ds = nn + ac - 1;
      if (owner_of(dd) == me) {
        const uint32_t lr = dd - r0;
        for (uint32_t w = tid; w < W; w += blockDim.x) ROW(lr)[w] = piv[w];
        if (tid == 0) ph[lr] = (uint8_t)pph;
      }
      if (owner_of(ds) == me) {
        const uint32_t lr = ds - r0;
        for (uint32_t w = tid; w < W; w += blockDim.x) ROW(lr)[w] = P[w];
        if (tid == 0) ph[lr] = (uint8_t)(rp >= 0 ? rp : (int32_t)pphase);
      }
      if (branch == 2) r += 1;
    }
    if (me == 0 && tid == 0) {
      a.anticom[j] = (int32_t)ac;
      a.result[j] = rp;
    }
    __syncthreads();
  }
  // write the rows back; every CTA is done with remote shared memory first
  cl.sync();
  for (uint32_t lr = warp; lr < nloc; lr += nwarps)
    for (uint32_t w = lane; w < W; w += 32) a.xzs[(size_t)(r0 + lr) * W + w] = ROW(lr)[w];
  for (uint32_t lr = tid; lr < nloc; lr += blockDim.x) a.ph[r0 + lr] = ph[lr];
  if (me == 0 && tid == 0) {
    if (a.kind == QCB_MIXED_STABILIZER || a.kind == QCB_MIXED_DESTABILIZER) *a.rank = r;
    a.status[0] = (int32_t)status;
    a.status[1] = (int32_t)jstop;
  }
}

static size_t proj_smem_bytes(uint32_t RB, uint32_t W) {
  return ((size_t)2 * W + 1 + (size_t)RB * (W + 1)) * 8 + 2 * (size_t)RB + 16 + 32 + 16 + 32 + 16;
}

// ---------------------------------------------------------------- the whole GPU
// project! of a Stabilizer / MixedStabilizer tableau too tall for one
// cluster's shared memory, on every SM: a cooperative grid (one CTA per SM,
// all resident) with two grid barriers per Pauli.  Phase 1: comm(pauli, row)
// for every row (warp per row) and the first anticommuting stabilizer row by
// a global atomicMin; barrier; phase 2: the same decision in every CTA, then
// row m <- pivot * row m for the anticommuting rows after the pivot (the
// loop of src/project_trace_reset.jl:296-305); barrier.  Writing the Pauli
// into the pivot row is deferred to the next Pauli's phase 1 (CTA 0), whose
// comm test takes that row from the Pauli kept in shared memory, so no third
// barrier is needed.  Every wait at a grid barrier is bounded: on expiry the
// CTA records QCB_ETIMEOUT and returns, and the others give up at their next
// barrier.
struct ProjGridArgs {
  ProjArgs a;
  uint32_t* bar;   // [0] arrivals, [1] generation
  uint32_t* gmin;  // [3]: the first anticommuting row of Pauli j at gmin[j % 3]
  int32_t* err;    // QCB_ETIMEOUT when a grid barrier wait gave up
  // test knob: CTA 1 leaves before the first barrier, so the others' waits
  // run out (0: off)
  uint32_t withhold;
};

// Bounded grid barrier; false when this CTA gave up waiting.
__device__ bool grid_barrier(uint32_t* bar, uint32_t nblocks, int32_t* err) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile uint32_t* gen = bar + 1;
    const uint32_t g0 = *gen;
    __threadfence();
    ok = 1;
    if (atomicAdd(bar, 1u) == nblocks - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      uint32_t it = 0;
      while (*gen == g0) {
        if (++it > (1u << 24)) {  // about a second
          ok = 0;
          atomicExch(err, QCB_ETIMEOUT);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

__global__ void __launch_bounds__(PROJ_THREADS) project_grid_kernel(const ProjGridArgs g) {
  const ProjArgs& a = g.a;
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const uint32_t G = gridDim.x, gw = blockIdx.x * nwarps + warp, NW = G * nwarps;
  const uint32_t W = a.W, len = W / 2, rows = a.rows;
  const bool lead = blockIdx.x == 0;
  extern __shared__ __align__(16) uint64_t smem[];
  uint64_t* Pb[2] = {smem, smem + W};  // the Pauli of projection j in Pb[j & 1]
  uint64_t* piv = smem + 2 * W;
  const uint32_t r = a.kind == QCB_STABILIZER ? rows : (uint32_t)*a.rank;
  uint32_t pprev = 0xFFFFFFFFu;  // the last pivot row, whose Pauli is not written yet
  uint8_t phprev = 0;
  uint32_t j = a.j0;
  for (; j < a.k; j++) {
    uint64_t* P = Pb[j & 1];
    const uint64_t* Pp = Pb[(j + 1) & 1];  // the previous Pauli
    const uint64_t* pj = a.paulis + (size_t)j * W;
    for (uint32_t w = tid; w < W; w += blockDim.x) P[w] = pj[w];
    __syncthreads();
    if (lead && pprev != 0xFFFFFFFFu) {
      for (uint32_t w = tid; w < W; w += blockDim.x) a.xzs[(size_t)pprev * W + w] = Pp[w];
      if (tid == 0) a.ph[pprev] = phprev;
    }
    if (lead && tid == 0) g.gmin[(j + 1) % 3] = 0xFFFFFFFFu;  // the slot of Pauli j + 1 (last used by j - 2)
    // 1. comm flags and the first anticommuting stabilizer row
    for (uint32_t m = gw; m < rows; m += NW) {
      const uint64_t* row = m == pprev ? Pp : a.xzs + (size_t)m * W;
      uint64_t acc = 0;
      for (uint32_t w = lane; w < len; w += 32) acc ^= (P[len + w] & row[w]) ^ (P[w] & row[len + w]);
      const uint32_t c = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)__popcll(acc)) & 1u;
      if (lane == 0) {
        a.flags[m] = (uint8_t)c;
        if (c && m < r) atomicMin(&g.gmin[j % 3], m);
      }
    }
    if (g.withhold && blockIdx.x == 1) return;
    if (!grid_barrier(g.bar, G, g.err)) return;
    // 2. the decision, the same in every CTA
    const uint32_t p = *(volatile uint32_t*)&g.gmin[j % 3];
    const int32_t rp = a.rand_ph ? (int32_t)a.rand_ph[j] : -1;
    if (p == 0xFFFFFFFFu) {
      // commutes with every stabilizer row
      pprev = 0xFFFFFFFFu;  // written in this Pauli's phase 1
      if (a.kind == QCB_STABILIZER && !a.keep_result) {
        if (lead && tid == 0) { a.anticom[j] = 0; a.result[j] = -1; }
        continue;  // phase 2 wrote nothing: no barrier needed
      }
      if (lead && tid == 0) { a.status[0] = PST_NEED_CANON; a.status[1] = (int32_t)j; }
      return;
    }
    for (uint32_t w = tid; w < W; w += blockDim.x) piv[w] = a.xzs[(size_t)p * W + w];
    __syncthreads();
    const uint32_t pph = a.ph[p];
    for (uint32_t m = p + 1 + gw; m < r; m += NW)
      if (a.flags[m]) warp_rowmul(a.xzs, a.ph, W, m, piv, pph, a.phases != 0, lane);
    if (lead && tid == 0) { a.anticom[j] = (int32_t)p + 1; a.result[j] = rp; }
    phprev = (uint8_t)(rp >= 0 ? rp : (int32_t)a.pph[j]);
    pprev = p;
    if (!grid_barrier(g.bar, G, g.err)) return;
  }
  if (lead && pprev != 0xFFFFFFFFu) {
    const uint64_t* Pp = Pb[(j + 1) & 1];
    for (uint32_t w = tid; w < W; w += blockDim.x) a.xzs[(size_t)pprev * W + w] = Pp[w];
    if (tid == 0) a.ph[pprev] = phprev;
  }
  if (lead && tid == 0) { a.status[0] = PST_OK; a.status[1] = (int32_t)a.k; }
}

static uint32_t g_proj_cs = 0;  // tuner override (0 = automatic)
static uint32_t g_proj_grid = 0;  // the whole-GPU kernel: 0 automatic, 1 always (where it applies), 2 never
static uint32_t g_proj_withhold = 0;  // test knob, see ProjGridArgs::withhold

}  // namespace qcb

using namespace qcb;

extern "C" {

// The k projections of one call: Paulis from a device tableau (pxzs, pph),
// or single-qubit Paulis (qubits: 1-based host array, basis bit 0 = X,
// bit 1 = Z); rand_host (host, 0 or 2 per projection) turns them into
// projectrand!.
static int project_impl(qcb_tableau* t, int kind, int32_t* rank_io, const uint64_t* pxzs, const uint8_t* pph,
                        const uint32_t* qubits, uint32_t basis, uint32_t k, int keep_result, int phases,
                        const uint8_t* rand_host, int32_t* anticom, int32_t* result, uint32_t* n_done, void* stream) {
  if (!t || !anticom || !result) return fail(QCB_EARG, "null argument");
  if (kind < 0 || kind > 3) return fail(QCB_EARG, "project!: bad state kind");
  const bool mixed = kind == QCB_MIXED_STABILIZER || kind == QCB_MIXED_DESTABILIZER;
  if (mixed && !rank_io) return fail(QCB_EARG, "project!: rank required for mixed states");
  if ((kind == QCB_DESTABILIZER || kind == QCB_MIXED_DESTABILIZER) && (t->rows % 2))
    return fail(QCB_EDIM, "project!: destabilizer tableaux have an even number of rows");
  if (kind == QCB_MIXED_DESTABILIZER && t->rows != 2 * t->nqubits)
    return fail(QCB_EDIM, "project!: MixedDestabilizer tableaux have 2n rows");
  if (mixed && (*rank_io < 0 || (uint32_t)*rank_io > (kind == QCB_MIXED_STABILIZER ? t->rows : t->rows / 2)))
    return fail(QCB_EBOUNDS, "project!: rank out of range");
  cudaStream_t st = S(stream);
  if (n_done) *n_done = 0;
  if (!k) return QCB_OK;
  const uint32_t W = t->W, len = W / 2;
  std::vector<uint32_t> q0;
  if (qubits) {
    q0.resize(k);
    for (uint32_t j = 0; j < k; j++) {
      if (qubits[j] == 0) return fail(QCB_EZEROQUBIT, "qubit indices start at 1 (NoZeroQubit)");
      if (qubits[j] > t->nqubits) return fail(QCB_EBOUNDS, "project: qubit index exceeds the state's qubits");
      q0[j] = qubits[j] - 1;
    }
  }
  // the Pauli of projection j in host memory (single-qubit mode)
  auto single_pauli = [&](uint32_t j) {
    std::vector<uint64_t> hp(W, 0);
    if (basis & 1u) hp[q0[j] >> 6] |= 1ull << (q0[j] & 63);
    if (basis & 2u) hp[len + (q0[j] >> 6)] |= 1ull << (q0[j] & 63);
    return hp;
  };
  uint32_t* d_q = nullptr;
  uint8_t* d_rand = nullptr;
  int32_t *d_anti = nullptr, *d_res = nullptr, *d_stat = nullptr, *d_rank = nullptr, *d_cout = nullptr;
  uint8_t* d_flags = nullptr;
  uint64_t* d_tmp = nullptr;
  uint8_t* d_tmpph = nullptr;
  QCB_CUDA(cudaMallocAsync(&d_anti, (size_t)k * 4, st));
  QCB_CUDA(cudaMallocAsync(&d_res, (size_t)k * 4, st));
  QCB_CUDA(cudaMallocAsync(&d_stat, 64, st));
  QCB_CUDA(cudaMallocAsync(&d_rank, 4, st));
  QCB_CUDA(cudaMallocAsync(&d_cout, 16, st));
  QCB_CUDA(cudaMallocAsync(&d_flags, std::max<uint32_t>(t->rows, 1), st));
  QCB_CUDA(cudaMallocAsync(&d_tmp, (size_t)t->W * 8 + 16, st));
  QCB_CUDA(cudaMallocAsync(&d_tmpph, 16, st));
  if (qubits) {
    QCB_CUDA(cudaMallocAsync(&d_q, (size_t)k * 4, st));
    QCB_CUDA(cudaMemcpyAsync(d_q, q0.data(), (size_t)k * 4, cudaMemcpyHostToDevice, st));
  }
  if (rand_host) {
    QCB_CUDA(cudaMallocAsync(&d_rand, k, st));
    QCB_CUDA(cudaMemcpyAsync(d_rand, rand_host, k, cudaMemcpyHostToDevice, st));
  }
  int32_t rank = mixed ? *rank_io : 0;
  QCB_CUDA(cudaMemcpyAsync(d_rank, &rank, 4, cudaMemcpyHostToDevice, st));

  // launch shape: the tableau in the cluster's shared memory when it fits
  // (the smallest cluster with at most 128 rows per CTA, or the tuned size),
  // else the rows stay in global memory
  const size_t maxsm = (size_t)device_max_smem_optin();
  uint32_t cs = 0, RB = 0;
  bool use_smem = false;
  for (uint32_t c = 1; c <= 16; c <<= 1) {
    if (g_proj_cs && c != g_proj_cs) continue;
    const uint32_t rb = (t->rows + c - 1) / c;
    if (proj_smem_bytes(rb, W) > maxsm) continue;
    cs = c; RB = rb; use_smem = true;
    if (g_proj_cs || rb <= 128) break;
  }
  const size_t sm = use_smem ? proj_smem_bytes(RB, W) : std::max<size_t>((size_t)2 * W * 8, 1024);
  if (!use_smem) cs = g_proj_cs ? g_proj_cs : 8;
  if (use_smem) {
    QCB_CUDA(cudaFuncSetAttribute(project_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, device_max_smem_optin()));
    if (cs > 8) QCB_CUDA(cudaFuncSetAttribute(project_smem_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  } else {
    QCB_CUDA(cudaFuncSetAttribute(project_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, device_max_smem_optin() - 1024));  // it has static shared memory too
    if (cs > 8) QCB_CUDA(cudaFuncSetAttribute(project_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  }
  // generic Paulis on a Stabilizer / MixedStabilizer tableau that does not
  // fit one cluster's shared memory: the whole GPU (project_grid_kernel)
  const size_t gsm = (size_t)3 * W * 8;
  const bool grid = g_proj_grid != 2 && !qubits && (kind == QCB_STABILIZER || kind == QCB_MIXED_STABILIZER) &&
                    (g_proj_grid == 1 || !use_smem) && gsm <= maxsm;
  uint32_t G = 0;
  uint32_t* d_bar = nullptr;  // [0..1] barrier, [2..4] first anticommuting rows, [5] timeout flag
  if (grid) {
    if (gsm > 48 * 1024)
      QCB_CUDA(cudaFuncSetAttribute(project_grid_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gsm));
    int nb = 0;
    QCB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, project_grid_kernel, PROJ_THREADS, gsm));
    G = (uint32_t)std::max(1, nb) * (uint32_t)std::max(device_sm_count(), 1);
    QCB_CUDA(cudaMallocAsync(&d_bar, 32, st));
  }
  int status = QCB_OK;
  uint32_t j0 = 0;
  std::vector<int32_t> h_anti(k, 0), h_res(k, -1);
  while (j0 < k) {
    ProjArgs a{};
    a.xzs = t->xzs; a.ph = t->phases; a.rows = t->rows; a.n = t->nqubits; a.W = t->W;
    a.kind = kind; a.rank = d_rank; a.paulis = pxzs; a.pph = pph;
    a.j0 = j0; a.k = k; a.keep_result = keep_result; a.phases = phases;
    a.anticom = d_anti; a.result = d_res; a.status = d_stat; a.flags = d_flags;
    a.qubits = d_q; a.basis = basis; a.rand_ph = d_rand;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(PROJ_THREADS);
    cfg.dynamicSmemBytes = sm;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int32_t htimeout = 0;
    if (grid) {
      QCB_CUDA(cudaMemsetAsync(d_bar, 0, 8, st));
      QCB_CUDA(cudaMemsetAsync(d_bar + 2, 0xFF, 12, st));
      QCB_CUDA(cudaMemsetAsync(d_bar + 5, 0, 4, st));
      QCB_CUDA(cudaMemsetAsync(d_stat, 0xFF, 8, st));
      ProjGridArgs ga{a, d_bar, d_bar + 2, (int32_t*)(d_bar + 5), G > 1 ? g_proj_withhold : 0u};
      void* args[] = {&ga};
      QCB_CUDA(cudaLaunchCooperativeKernel((const void*)project_grid_kernel, dim3(G), dim3(PROJ_THREADS), args, gsm,
                                           st));
    } else if (use_smem) {
      ProjSmemArgs pa{a, RB};
      QCB_CUDA(cudaLaunchKernelEx(&cfg, project_smem_kernel, pa));
    } else {
      QCB_CUDA(cudaLaunchKernelEx(&cfg, project_kernel, a));
    }
    QCB_LAUNCHED();
    int32_t hs[2];
    QCB_CUDA(cudaMemcpyAsync(hs, d_stat, 8, cudaMemcpyDeviceToHost, st));
    if (grid) QCB_CUDA(cudaMemcpyAsync(&htimeout, d_bar + 5, 4, cudaMemcpyDeviceToHost, st));
    QCB_CUDA(cudaStreamSynchronize(st));
    if (htimeout) {
      status = fail(QCB_ETIMEOUT, "project!: a grid barrier wait of the whole-GPU kernel expired");
      break;
    }
    if (hs[0] == PST_OK) break;
    const uint32_t j = (uint32_t)hs[1];
    if (hs[0] == PST_BADSTRUCT) {
      status = fail(QCB_EBADSTRUCT,
                    "`Destabilizer` can not efficiently (faster than n^3) detect whether you are projecting on a "
                    "stabilized or a logical operator. Switch to one of the `Mixed*` data structures.");
      if (n_done) *n_done = j;
      j0 = k;
      break;
    }
    // PST_NEED_CANON: canonicalize the stabilizer view, then generate!
    int32_t r_now = rank;
    if (kind == QCB_MIXED_STABILIZER) QCB_CUDA(cudaMemcpy(&r_now, d_rank, 4, cudaMemcpyDeviceToHost));
    const uint32_t nr = kind == QCB_STABILIZER ? t->rows : (uint32_t)r_now;
    if (int s = canonicalize_view(t->xzs, t->phases, nr, t->nqubits, t->W, phases, d_cout, st)) { status = s; break; }
    std::vector<uint64_t> hp;
    const uint8_t zero = 0;
    if (qubits) {
      hp = single_pauli(j);
      QCB_CUDA(cudaMemcpyAsync(d_tmp, hp.data(), (size_t)W * 8, cudaMemcpyHostToDevice, st));
      QCB_CUDA(cudaMemcpyAsync(d_tmpph, &zero, 1, cudaMemcpyHostToDevice, st));
    } else {
      QCB_CUDA(cudaMemcpyAsync(d_tmp, pxzs + (size_t)j * W, (size_t)W * 8, cudaMemcpyDeviceToDevice, st));
      QCB_CUDA(cudaMemcpyAsync(d_tmpph, pph + j, 1, cudaMemcpyDeviceToDevice, st));
    }
    if (int s = generate_dev(d_tmp, d_tmpph, t->xzs, t->phases, nr, t->W, phases, d_cout + 2, nullptr, 0,
                             (uint32_t*)(d_cout + 3), st)) { status = s; break; }
    int32_t cout[4];
    uint8_t gph = 0;
    QCB_CUDA(cudaMemcpyAsync(cout, d_cout, 16, cudaMemcpyDeviceToHost, st));
    QCB_CUDA(cudaMemcpyAsync(&gph, d_tmpph, 1, cudaMemcpyDeviceToHost, st));
    QCB_CUDA(cudaStreamSynchronize(st));
    int32_t anti = 0, res = -1;
    if (cout[2]) {
      res = gph;
    } else {
      anti = cout[1] + 1;
      if (kind == QCB_MIXED_STABILIZER && anti == r_now + 1) {
        // ms.tab[rank+1] = pauli; rank += 1  (src/project_trace_reset.jl:310-317)
        if ((uint32_t)r_now >= t->rows) { status = fail(QCB_EBOUNDS, "MixedStabilizer tableau is full"); break; }
        if (qubits) {
          QCB_CUDA(cudaMemcpyAsync(t->xzs + (size_t)r_now * W, hp.data(), (size_t)W * 8, cudaMemcpyHostToDevice, st));
          QCB_CUDA(cudaMemcpyAsync(t->phases + r_now, &zero, 1, cudaMemcpyHostToDevice, st));
        } else {
          QCB_CUDA(cudaMemcpyAsync(t->xzs + (size_t)r_now * W, pxzs + (size_t)j * W, (size_t)W * 8,
                                   cudaMemcpyDeviceToDevice, st));
          QCB_CUDA(cudaMemcpyAsync(t->phases + r_now, pph + j, 1, cudaMemcpyDeviceToDevice, st));
        }
        r_now += 1;
        QCB_CUDA(cudaMemcpyAsync(d_rank, &r_now, 4, cudaMemcpyHostToDevice, st));
      }
      if (rand_host && anti > 0) {
        // projectrand!: the new stabilizer row anti gets a random sign
        if ((uint32_t)anti > t->rows) { status = fail(QCB_EBOUNDS, "projectrand!: no stabilizer row to randomize"); break; }
        QCB_CUDA(cudaMemcpyAsync(t->phases + (anti - 1), rand_host + j, 1, cudaMemcpyHostToDevice, st));
        res = rand_host[j];
      }
    }
    QCB_CUDA(cudaMemcpyAsync(d_anti + j, &anti, 4, cudaMemcpyHostToDevice, st));
    QCB_CUDA(cudaMemcpyAsync(d_res + j, &res, 4, cudaMemcpyHostToDevice, st));
    QCB_CUDA(cudaStreamSynchronize(st));
    j0 = j + 1;
  }
  if (status == QCB_OK || status == QCB_EBADSTRUCT) {
    QCB_CUDA(cudaMemcpyAsync(h_anti.data(), d_anti, (size_t)k * 4, cudaMemcpyDeviceToHost, st));
    QCB_CUDA(cudaMemcpyAsync(h_res.data(), d_res, (size_t)k * 4, cudaMemcpyDeviceToHost, st));
    if (mixed) QCB_CUDA(cudaMemcpyAsync(&rank, d_rank, 4, cudaMemcpyDeviceToHost, st));
    QCB_CUDA(cudaStreamSynchronize(st));
    std::copy(h_anti.begin(), h_anti.end(), anticom);
    std::copy(h_res.begin(), h_res.end(), result);
    if (mixed) *rank_io = rank;
    if (status == QCB_OK && n_done) *n_done = k;
  }
  cudaFreeAsync(d_anti, st); cudaFreeAsync(d_res, st); cudaFreeAsync(d_stat, st);
  cudaFreeAsync(d_rank, st); cudaFreeAsync(d_cout, st); cudaFreeAsync(d_flags, st);
  cudaFreeAsync(d_tmp, st); cudaFreeAsync(d_tmpph, st);
  if (d_q) cudaFreeAsync(d_q, st);
  if (d_rand) cudaFreeAsync(d_rand, st);
  if (d_bar) cudaFreeAsync(d_bar, st);
  cudaStreamSynchronize(st);
  return status;
}

int qcb_project(qcb_tableau* t, int kind, int32_t* rank_io, const qcb_tableau* paulis, int keep_result,
                int phases, int32_t* anticom, int32_t* result, uint32_t* n_done, void* stream) {
  if (!t || !paulis) return fail(QCB_EARG, "null argument");
  if (paulis->nqubits != t->nqubits) return fail(QCB_EDIM, "project!: the Pauli and the state act on different numbers of qubits");
  return project_impl(t, kind, rank_io, paulis->xzs, paulis->phases, nullptr, 0, paulis->rows, keep_result, phases,
                      nullptr, anticom, result, n_done, stream);
}

int qcb_project_qubit(qcb_tableau* t, int kind, int32_t* rank_io, uint32_t basis, const uint32_t* qubits, size_t k,
                      int keep_result, int phases, int32_t* anticom, int32_t* result, uint32_t* n_done,
                      void* stream) {
  if (basis < 1 || basis > 3) return fail(QCB_EARG, "project: basis is 1 (X), 2 (Z) or 3 (Y)");
  if (k && !qubits) return fail(QCB_EARG, "null argument");
  if (k > 0xFFFFFFFFull) return fail(QCB_EARG, "too many projections");
  return project_impl(t, kind, rank_io, nullptr, nullptr, qubits, basis, (uint32_t)k, keep_result, phases, nullptr,
                      anticom, result, n_done, stream);
}

int qcb_projectrand(qcb_tableau* t, int kind, int32_t* rank_io, const qcb_tableau* paulis, uint32_t basis,
                    const uint32_t* qubits, size_t k, const uint8_t* rand_phases, int32_t* anticom, int32_t* result,
                    uint32_t* n_done, void* stream) {
  if (!rand_phases) return fail(QCB_EARG, "null argument");
  if (paulis) {
    if (paulis->nqubits != t->nqubits) return fail(QCB_EDIM, "project!: the Pauli and the state act on different numbers of qubits");
    for (uint32_t j = 0; j < paulis->rows; j++)
      if (rand_phases[j] != 0 && rand_phases[j] != 2) return fail(QCB_EARG, "projectrand!: random phases are 0 or 2");
    return project_impl(t, kind, rank_io, paulis->xzs, paulis->phases, nullptr, 0, paulis->rows, 1, 1, rand_phases,
                        anticom, result, n_done, stream);
  }
  if (basis < 1 || basis > 3) return fail(QCB_EARG, "project: basis is 1 (X), 2 (Z) or 3 (Y)");
  if (k && !qubits) return fail(QCB_EARG, "null argument");
  for (size_t j = 0; j < k; j++)
    if (rand_phases[j] != 0 && rand_phases[j] != 2) return fail(QCB_EARG, "projectrand!: random phases are 0 or 2");
  return project_impl(t, kind, rank_io, nullptr, nullptr, qubits, basis, (uint32_t)k, 1, 1, rand_phases, anticom,
                      result, n_done, stream);
}

}  // extern "C"

namespace qcb {
void set_project_cluster(uint32_t cs) { g_proj_cs = cs; }
void set_project_grid(uint32_t v) { g_proj_grid = v; }
void set_project_withhold(uint32_t v) { g_proj_withhold = v; }
}
