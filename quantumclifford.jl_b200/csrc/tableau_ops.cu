// tableau_ops.cu -- row algebra on device tableaux.
//
//  mul_left!  (src/mul_leftright.jl:75-142, 171-229): r <- l * r with the
//             phase of the product.  The phase is the sum over bit lanes of
//             independent mod-4 counters (cnt1 = low bit, cnt2 = high bit),
//             so any partition of the words into threads sums exactly:
//             phase = (sum popc(cnt1) + 2 * sum popc(cnt2)) mod 4.
//  prodphase / comm (src/QuantumClifford.jl:723-859).
//  symbolic gates with phases (src/symbolic_cliffords.jl:62-74, 293-316).
//  dense apply! (src/dense_cliffords.jl:135-169).
#include <algorithm>
#include <mutex>

#include "qcb_internal.h"

namespace qcb {

// Stim phase-counter step on one word pair (src/mul_leftright.jl:90-96).
template <class T>
__device__ __forceinline__ void mul_step(T x1, T z1, T& x2, T& z2, uint64_t& c1, uint64_t& c2) {
  const uint64_t nx = x1 ^ x2, nz = z1 ^ z2;
  const uint64_t x1z2 = (uint64_t)x1 & (uint64_t)z2;
  const uint64_t anti = ((uint64_t)x2 & (uint64_t)z1) ^ x1z2;
  c2 ^= (c1 ^ nx ^ nz ^ x1z2) & anti;
  c1 ^= anti;
  x2 = (T)nx;
  z2 = (T)nz;
}

__device__ __forceinline__ uint32_t cnt_phase(uint64_t c1, uint64_t c2) {
  return (uint32_t)(__popcll(c1) + 2 * __popcll(c2));
}

// mul_right!(l, r) runs the word steps of mul_left!(l <- r * l) and adds
// twice the anticommutation count (src/mul_leftright.jl:128-131): phase
// (rcnt1 + 2 rcnt2) + 2 rcnt1, i.e. 3 popc(cnt1) + 2 popc(cnt2) per lane.
template <bool RIGHT>
__device__ __forceinline__ uint32_t lane_phase(uint64_t c1, uint64_t c2) {
  return RIGHT ? (uint32_t)(3 * __popcll(c1) + 2 * __popcll(c2)) : cnt_phase(c1, c2);
}

// Grid-stride mul_left! over two long Paulis.  VEC = 2 uses 128-bit loads
// (needs len even and 16-byte aligned halves).  Each block adds its phase
// sum (mod 4) into acc[0] and counts itself done in acc[1]; the last block
// to finish writes r.phase <- (s + r.phase + l.phase) & 3
// (src/mul_leftright.jl:140) and clears both, so one launch does the call.
template <int VEC, bool PH, bool RIGHT = false>
__global__ void __launch_bounds__(256) mul_left_long_kernel(uint64_t* __restrict__ r,
                                                            const uint64_t* __restrict__ l,
                                                            uint64_t len, uint32_t* acc,
                                                            uint8_t* r_phase, const uint8_t* l_phase) {
  uint64_t c1a = 0, c2a = 0, c1b = 0, c2b = 0;
  const uint64_t nvec = len / VEC;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nvec; i += stride) {
    if (VEC == 2) {
      const ulonglong2 lx = __ldcs((const ulonglong2*)l + i);
      const ulonglong2 lz = __ldcs((const ulonglong2*)(l + len) + i);
      ulonglong2 rx = __ldcs((const ulonglong2*)r + i);
      ulonglong2 rz = __ldcs((const ulonglong2*)(r + len) + i);
      if (PH) {
        mul_step(lx.x, lz.x, rx.x, rz.x, c1a, c2a);
        mul_step(lx.y, lz.y, rx.y, rz.y, c1b, c2b);
      } else {
        rx.x ^= lx.x; rx.y ^= lx.y; rz.x ^= lz.x; rz.y ^= lz.y;
      }
      __stcs((ulonglong2*)r + i, rx);
      __stcs((ulonglong2*)(r + len) + i, rz);
    } else {
      const uint64_t lx = __ldcs(l + i), lz = __ldcs(l + len + i);
      uint64_t rx = __ldcs(r + i), rz = __ldcs(r + len + i);
      if (PH) mul_step(lx, lz, rx, rz, c1a, c2a);
      else { rx ^= lx; rz ^= lz; }
      __stcs(r + i, rx);
      __stcs(r + len + i, rz);
    }
  }
  if (!PH) return;
  uint32_t v = (lane_phase<RIGHT>(c1a, c2a) + lane_phase<RIGHT>(c1b, c2b)) & 3u;
  v = __reduce_add_sync(0xFFFFFFFFu, v) & 3u;
  __shared__ uint32_t wsum[32];
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) wsum[wid] = v;
  __syncthreads();
  if (wid == 0) {
    uint32_t s = lane < (blockDim.x >> 5) ? wsum[lane] : 0u;
    s = __reduce_add_sync(0xFFFFFFFFu, s) & 3u;
    if (lane == 0) {
      if (s) atomicAdd(acc, s);
      __threadfence();
      if (atomicAdd(acc + 1, 1u) == gridDim.x - 1) {  // the last block
        __threadfence();
        const uint32_t tot = atomicExch(acc, 0u) & 3u;
        atomicExch(acc + 1, 0u);
        r_phase[0] = (uint8_t)((tot + r_phase[0] + l_phase[0]) & 3u);
      }
    }
  }
}

// r.phase <- (s + r.phase + l.phase) & 3 (src/mul_leftright.jl:140); clears acc.
__global__ void mul_left_finish_kernel(uint8_t* r_phase, const uint8_t* l_phase, uint32_t* acc,
                                       int phases) {
  const uint32_t s = acc[0] & 3u;
  if (phases) r_phase[0] = (uint8_t)((s + r_phase[0] + l_phase[0]) & 3u);
  acc[0] = 0;
}

// Row-level ops: one warp per target row; lanes stride over the words.
template <bool PH>
__device__ __forceinline__ uint32_t warp_mul_left_row(uint64_t* r, const uint64_t* l, uint32_t len,
                                                      uint32_t lane) {
  uint64_t c1 = 0, c2 = 0;
  for (uint32_t w = lane; w < len; w += 32) {
    uint64_t rx = r[w], rz = r[len + w];
    const uint64_t lx = l[w], lz = l[len + w];
    if (PH) mul_step(lx, lz, rx, rz, c1, c2);
    else { rx ^= lx; rz ^= lz; }
    r[w] = rx;
    r[len + w] = rz;
  }
  if (!PH) return 0;
  return __reduce_add_sync(0xFFFFFFFFu, cnt_phase(c1, c2) & 3u) & 3u;
}

// mul_left!(s::Tableau, p::PauliOperator) (src/mul_leftright.jl:221-227).
__global__ void mul_left_tab_pauli_kernel(uint64_t* xzs, uint8_t* ph, uint32_t rows, uint32_t W,
                                          const uint64_t* p, const uint8_t* pph, int phases) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= rows) return;
  uint64_t* r = xzs + (uint64_t)warp * W;
  if (phases) {
    const uint32_t s = warp_mul_left_row<true>(r, p, W / 2, lane);
    if (lane == 0) ph[warp] = (uint8_t)((s + ph[warp] + pph[0]) & 3u);
  } else {
    warp_mul_left_row<false>(r, p, W / 2, lane);
  }
}

// mul_left!(s::Tableau, m, i) (src/mul_leftright.jl:177-181), 0-based rows.
__global__ void mul_left_row_kernel(uint64_t* xzs, uint8_t* ph, uint32_t W, uint32_t m, uint32_t i,
                                    int phases) {
  const uint32_t lane = threadIdx.x & 31;
  if (threadIdx.x >= 32) return;
  uint64_t* r = xzs + (uint64_t)m * W;
  const uint64_t* l = xzs + (uint64_t)i * W;
  if (phases) {
    const uint32_t s = warp_mul_left_row<true>(r, l, W / 2, lane);
    if (lane == 0) ph[m] = (uint8_t)((s + ph[m] + ph[i]) & 3u);
  } else {
    warp_mul_left_row<false>(r, l, W / 2, lane);
  }
}

// The mul_left!/mul_right! family on rows (src/mul_leftright.jl:137-245,
// ext/QuantumCliffordKAExt/mul_leftright.jl:101-460): one warp per target row
// a = s_row + k, source row b = t_row + k * t_step; the added phase is
// add_ph[b] (t's phases, or s's for the reference's cross-tableau methods).
template <bool RIGHT, bool PH>
__global__ void __launch_bounds__(256) mul_rows_kernel(uint64_t* s_xz, uint8_t* s_ph, uint32_t s_row,
                                                       uint32_t count, const uint64_t* t_xz, uint32_t t_row,
                                                       uint32_t t_step, uint32_t W, const uint8_t* add_ph) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t len = W / 2;
  for (uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < count; k += nwarps) {
    const uint32_t a = s_row + k, b = t_row + k * t_step;
    uint64_t* r = s_xz + (uint64_t)a * W;
    const uint64_t* l = t_xz + (uint64_t)b * W;
    uint64_t c1 = 0, c2 = 0;
    for (uint32_t w = lane; w < len; w += 32) {
      uint64_t rx = r[w], rz = r[len + w];
      const uint64_t lx = l[w], lz = l[len + w];
      if (PH) mul_step(lx, lz, rx, rz, c1, c2);
      else { rx ^= lx; rz ^= lz; }
      r[w] = rx;
      r[len + w] = rz;
    }
    if (PH) {
      const uint32_t v = __reduce_add_sync(0xFFFFFFFFu, lane_phase<RIGHT>(c1, c2) & 3u) & 3u;
      if (lane == 0) s_ph[a] = (uint8_t)((v + s_ph[a] + add_ph[b]) & 3u);
    }
  }
}

// prodphase (src/QuantumClifford.jl:723-733) and comm (:791-798) of two rows.
__global__ void prodphase_comm_kernel(const uint64_t* l, uint8_t lph, const uint64_t* r, uint8_t rph,
                                      uint32_t len, int what, uint8_t* out) {
  const uint32_t lane = threadIdx.x & 31;
  if (threadIdx.x >= 32) return;
  int32_t acc = 0;
  uint64_t cm = 0;
  for (uint32_t w = lane; w < len; w += 32) {
    const uint64_t x1 = l[w], x2 = r[w], z1 = l[len + w], z2 = r[len + w];
    acc += __popcll((~z2 & x2 & ~x1 & z1) | (z2 & ~x2 & x1 & z1) | (z2 & x2 & x1 & ~z1));
    acc -= __popcll((z2 & x2 & ~x1 & z1) | (~z2 & x2 & x1 & z1) | (z2 & ~x2 & x1 & ~z1));
    cm ^= (z1 & x2) ^ (x1 & z2);
  }
  const int32_t tot = __reduce_add_sync(0xFFFFFFFFu, acc);
  const uint32_t par = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)__popcll(cm)) & 1u;
  if (lane == 0) {
    if (what == 0) out[0] = (uint8_t)(((uint32_t)tot + lph + rph) & 3u);
    else out[0] = (uint8_t)par;
  }
}

// ---------------------------------------------------------- symbolic gates
// Bit-sliced truth tables with the phase flag (src/symbolic_cliffords.jl
// :105-118 and :358-395).
__device__ __forceinline__ uint64_t g1(uint32_t op, uint64_t& x, uint64_t& z) {
  const uint64_t X = x, Z = z;
  if ((op & 0xFFu) == QCB_OP_SQO) {
    // SingleQubitOperator (src/symbolic_cliffords.jl:178-206), flags in bits
    // 8..13: +2 for px & x, for pz & z, and for x & z when the map sends Y to
    // minus the product of the images of X and Z
    const uint32_t f = op >> 8;
    const bool bxx = f & 1u, bxz = f & 2u, bzx = f & 4u, bzz = f & 8u;
    const uint64_t xx = 0ull - (uint64_t)bxx, xz = 0ull - (uint64_t)bxz;
    const uint64_t zx = 0ull - (uint64_t)bzx, zz = 0ull - (uint64_t)bzz;
    const bool anticom = (!bzz && bxz && !bxx && bzx) || (bzz && !bxz && bxx && bzx) || (bzz && bxz && bxx && !bzx);
    x = (X & xx) ^ (Z & zx);
    z = (X & xz) ^ (Z & zz);
    return ((f & 16u) ? X : 0ull) ^ ((f & 32u) ? Z : 0ull) ^ (anticom ? (X & Z) : 0ull);
  }
  switch (op) {
    case QCB_OP_H: x = Z; z = X; return X & Z;
    case QCB_OP_HXY: z = X ^ Z; return ~X & Z;
    case QCB_OP_HYZ: x = X ^ Z; return X & ~Z;
    case QCB_OP_S: z = X ^ Z; return X & Z;
    case QCB_OP_SDAG: z = X ^ Z; return X & ~Z;
    case QCB_OP_X: return Z;
    case QCB_OP_Y: return X ^ Z;
    case QCB_OP_Z: return X;
    case QCB_OP_SQRTX: x = X ^ Z; return ~X & Z;
    case QCB_OP_INVSQRTX: x = X ^ Z; return X & Z;
    case QCB_OP_SQRTY: x = Z; z = X; return X & ~Z;
    case QCB_OP_INVSQRTY: x = Z; z = X; return Z & ~X;
    case QCB_OP_CXYZ: x = X ^ Z; z = X; return 0;
    case QCB_OP_CZYX: x = Z; z = X ^ Z; return 0;
    default: return 0;
  }
}

__device__ __forceinline__ uint64_t g2(uint32_t op, uint64_t& x1, uint64_t& z1, uint64_t& x2,
                                       uint64_t& z2) {
  const uint64_t a = x1, b = z1, c = x2, d = z2;
  switch (op) {
    case QCB_OP_SWAP: x1 = c; z1 = d; x2 = a; z2 = b; return 0;
    case QCB_OP_CNOT: z1 = b ^ d; x2 = c ^ a; return (a & b & c & d) | (a & d & ~(b | c));
    case QCB_OP_CPHASE: z1 = b ^ c; z2 = d ^ a; return (a & b & c & ~d) | (a & ~b & c & d);
    case QCB_OP_ZCX: z1 = b ^ d; x2 = c ^ a; return (a & d) & ~(b ^ c);
    case QCB_OP_ZCY: z1 = c ^ b ^ d; x2 = c ^ a; z2 = d ^ a; return a & (c ^ b) & (c ^ d);
    case QCB_OP_ZCZ: z1 = b ^ c; z2 = d ^ a; return (b ^ d) & (a & c);
    case QCB_OP_XCX: x1 = d ^ a; x2 = c ^ b; return (b & d) & (a ^ c);
    case QCB_OP_XCY: x1 = a ^ c ^ d; x2 = b ^ c; z2 = d ^ b; return b & (c ^ d) & ~(c ^ a);
    case QCB_OP_XCZ: x1 = a ^ c; z2 = d ^ b; return (c & b) & ~(a ^ d);
    case QCB_OP_YCX: x1 = a ^ d; z1 = d ^ b; x2 = a ^ b ^ c; return d & (a ^ b) & ~(c ^ a);
    case QCB_OP_YCY:
      x1 = a ^ d ^ c; z1 = b ^ c ^ d; x2 = a ^ c ^ b; z2 = a ^ b ^ d;
      return (a & ~b & ~c & d) | (~a & b & c & ~d);
    case QCB_OP_YCZ: x1 = a ^ c; z1 = c ^ b; z2 = d ^ a ^ b; return c & (a ^ b) & (d ^ a);
    case QCB_OP_SWAPCX:
      x1 = c; z1 = d ^ b; x2 = c ^ a; z2 = b;
      return (a & b & c & d) | (~a & b & c & ~d);
    case QCB_OP_INVSWAPCX:
      x1 = c ^ a; z1 = d; x2 = a; z2 = d ^ b;
      return (a & b & c & d) | (a & ~b & ~c & d);
    case QCB_OP_ISWAP:
      x1 = c; z1 = a ^ d ^ c; x2 = a; z2 = a ^ c ^ b;
      return (a & b & ~c) | (~a & c & d);
    case QCB_OP_INVISWAP:
      x1 = c; z1 = a ^ d ^ c; x2 = a; z2 = a ^ c ^ b;
      return (a & ~b & ~c) | (~a & c & ~d);
    case QCB_OP_CZSWAP:
      x1 = c; z1 = d ^ a; x2 = a; z2 = c ^ b;
      return (a & ~b & c & d) | (a & b & c & ~d);
    case QCB_OP_CXSWAP:
      x1 = c ^ a; z1 = d; x2 = a; z2 = d ^ b;
      return (a & ~b & ~c & d) | (a & b & c & d);
    case QCB_OP_ZCRY:
      z1 = a ^ b ^ c ^ d; x2 = a ^ c; z2 = a ^ d;
      return (a & ~b & c) | (a & ~b & ~d) | (a & c & ~d);
    case QCB_OP_INVZCRY:
      z1 = a ^ b ^ c ^ d; x2 = a ^ c; z2 = a ^ d;
      return (a & b & ~c) | (a & b & d) | (a & ~c & d);
    case QCB_OP_SQRTZZ:
      z1 = a ^ c ^ b; z2 = a ^ d ^ c;
      return (a & b & ~c) | (~a & c & d);
    case QCB_OP_INVSQRTZZ:
      z1 = a ^ c ^ b; z2 = a ^ d ^ c;
      return (a & ~b & ~c) | (~a & c & ~d);
    case QCB_OP_SQRTXX:
      x1 = b ^ d ^ a; x2 = b ^ c ^ d;
      return (~a & b & ~d) | (~b & ~c & d);
    case QCB_OP_INVSQRTXX:
      x1 = b ^ d ^ a; x2 = b ^ c ^ d;
      return (a & b & ~d) | (~b & c & d);
    case QCB_OP_SQRTYY:
      x1 = b ^ c ^ d; z1 = a ^ d ^ c; x2 = a ^ b ^ d; z2 = a ^ c ^ b;
      return (~a & ~b & c & ~d) | (a & ~b & ~c & ~d) | (a & ~b & c & d) | (a & b & c & ~d);
    case QCB_OP_INVSQRTYY:
      x1 = b ^ c ^ d; z1 = a ^ d ^ c; x2 = a ^ b ^ d; z2 = a ^ c ^ b;
      return (a & b & ~c & d) | (~a & b & c & d) | (~a & b & ~c & ~d) | (~a & ~b & ~c & d);
    default: return 0;
  }
}

struct GateOp {
  uint32_t op, q1, q2, pad;
};
// Gates passed to one launch by value (kernel parameter space, 2 KB), so a
// gate list needs no device allocation, no copy and no synchronisation.
constexpr uint32_t GATE_BATCH = 128;
struct GateBatch {
  GateOp op[GATE_BATCH];
};

// Thread per row; the batch's gates are applied to that row in order.  The
// launch may be a programmatic dependent of the launch before it on the
// stream: the dependents of this one are released at once, and the rows are
// touched only after griddepcontrol.wait (the predecessor has completed and
// its writes are visible; a no-op for a plain launch).
__global__ void apply_gates_kernel(uint64_t* xzs, uint8_t* ph, uint32_t rows, uint32_t W,
                                   const __grid_constant__ GateBatch ops, uint32_t nops, int phases) {
  asm volatile("griddepcontrol.launch_dependents;");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  uint64_t* row = xzs + (uint64_t)r * W;
  const uint32_t len = W / 2;
  uint32_t p = ph[r];
  for (uint32_t k = 0; k < nops; k++) {
    const GateOp g = ops.op[k];
    if ((g.op & 0xFFu) < QCB_OP_CNOT) {  // SingleQubitOperator carries flags above bit 8
      const uint32_t q = g.q1, w = q >> 6, s = q & 63;
      uint64_t x = (row[w] >> s) & 1, z = (row[len + w] >> s) & 1;
      const uint64_t f = g1(g.op, x, z) & 1;
      row[w] = (row[w] & ~(1ull << s)) | ((x & 1) << s);
      row[len + w] = (row[len + w] & ~(1ull << s)) | ((z & 1) << s);
      if (phases && f) p = (p + 2) & 3;
    } else {
      const uint32_t w1 = g.q1 >> 6, s1 = g.q1 & 63, w2 = g.q2 >> 6, s2 = g.q2 & 63;
      uint64_t x1 = (row[w1] >> s1) & 1, z1 = (row[len + w1] >> s1) & 1;
      uint64_t x2 = (row[w2] >> s2) & 1, z2 = (row[len + w2] >> s2) & 1;
      const uint64_t f = g2(g.op, x1, z1, x2, z2) & 1;
      row[w1] = (row[w1] & ~(1ull << s1)) | ((x1 & 1) << s1);
      row[len + w1] = (row[len + w1] & ~(1ull << s1)) | ((z1 & 1) << s1);
      row[w2] = (row[w2] & ~(1ull << s2)) | ((x2 & 1) << s2);
      row[len + w2] = (row[len + w2] & ~(1ull << s2)) | ((z2 & 1) << s2);
      if (phases && f) p = (p + 2) & 3;
    }
  }
  ph[r] = (uint8_t)p;
}

// ---------------------------------------------------------- dense apply!
// One warp per state row.  The ordered product over qubits of the Clifford's
// images (src/dense_cliffords.jl:152-169) is accumulated in registers; the
// phase counters run across all the multiplications (each multiplication adds
// +-1 per anticommuting lane, independent of the current counter value), so
// one reduction at the end gives the exact total.
template <int MAXW>
__global__ void __launch_bounds__(256) apply_dense_kernel(uint64_t* xzs, uint8_t* ph, uint32_t rows,
                                                          uint32_t W, uint32_t n,
                                                          const uint64_t* __restrict__ c,
                                                          const uint8_t* __restrict__ cph,
                                                          int phases) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= rows) return;
  const uint32_t len = W / 2;
  constexpr int PER = (MAXW / 2 + 31) / 32;  // words per lane per half
  uint64_t bx[PER], bz[PER], c1[PER], c2[PER];
#pragma unroll
  for (int k = 0; k < PER; k++) { bx[k] = bz[k] = c1[k] = c2[k] = 0; }
  uint64_t* row = xzs + (uint64_t)warp * W;
  uint32_t extra = 0;  // sum of Clifford-row phases and -1 corrections (mod 4)
  for (uint32_t wq = 0; wq < len; wq++) {
    const uint64_t xw = row[wq], zw = row[len + wq];  // broadcast loads
    uint64_t both = xw | zw;
    while (both) {
      const uint32_t b = __ffsll((long long)both) - 1;
      both &= both - 1;
      const uint32_t q = wq * 64 + b;
      if (q >= n) break;
      const bool x = (xw >> b) & 1, z = (zw >> b) & 1;
      if (x && z) extra += 3;  // phase -= 1
      if (x) {
        const uint64_t* cr = c + (uint64_t)q * W;
#pragma unroll
        for (int k = 0; k < PER; k++) {
          const uint32_t w = lane + 32 * k;
          if (w < len) mul_step<uint64_t>(__ldg(cr + w), __ldg(cr + len + w), bx[k], bz[k], c1[k], c2[k]);
        }
        extra += cph[q];
      }
      if (z) {
        const uint64_t* cr = c + (uint64_t)(q + n) * W;
#pragma unroll
        for (int k = 0; k < PER; k++) {
          const uint32_t w = lane + 32 * k;
          if (w < len) mul_step<uint64_t>(__ldg(cr + w), __ldg(cr + len + w), bx[k], bz[k], c1[k], c2[k]);
        }
        extra += cph[q + n];
      }
    }
  }
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < PER; k++) s += cnt_phase(c1[k], c2[k]);
  s = __reduce_add_sync(0xFFFFFFFFu, s & 3u) & 3u;
  __syncwarp();
#pragma unroll
  for (int k = 0; k < PER; k++) {
    const uint32_t w = lane + 32 * k;
    if (w < len) { row[w] = bx[k]; row[len + w] = bz[k]; }
  }
  if (lane == 0) ph[warp] = phases ? (uint8_t)((s + extra + ph[warp]) & 3u) : (uint8_t)0;
}

// The same product split over G warps per state row (one row per CTA): warp g
// multiplies the Clifford rows of its share of the qubit words in order into
// a partial product (bits, counters, phase), and warp 0 then left-multiplies
// the partials in order.  The Pauli product is associative with exact phases,
// so P_{G-1} ... P_1 P_0 is the ordered product of all the images, and the
// row gets G times the warps of the one-warp kernel.
template <int MAXW, int G>
__global__ void __launch_bounds__(32 * G) apply_dense_split_kernel(uint64_t* xzs, uint8_t* ph, uint32_t rows,
                                                                  uint32_t W, uint32_t n,
                                                                  const uint64_t* __restrict__ c,
                                                                  const uint8_t* __restrict__ cph, int phases) {
  __shared__ uint64_t part[G][MAXW];
  __shared__ uint32_t pph[G];
  const uint32_t r = blockIdx.x, g = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (r >= rows) return;
  const uint32_t len = W / 2;
  constexpr int PER = (MAXW / 2 + 31) / 32;  // words per lane per half
  uint64_t bx[PER], bz[PER], c1[PER], c2[PER];
#pragma unroll
  for (int k = 0; k < PER; k++) { bx[k] = bz[k] = c1[k] = c2[k] = 0; }
  uint64_t* row = xzs + (uint64_t)r * W;
  uint32_t extra = 0;  // Clifford-row phases and the -1 of every Y (mod 4)
  const uint32_t wq0 = g * len / G, wq1 = (g + 1) * len / G;
  for (uint32_t wq = wq0; wq < wq1; wq++) {
    const uint64_t xw = row[wq], zw = row[len + wq];  // broadcast loads
    uint64_t both = xw | zw;
    while (both) {
      const uint32_t b = __ffsll((long long)both) - 1;
      both &= both - 1;
      const uint32_t q = wq * 64 + b;
      if (q >= n) break;
      const bool x = (xw >> b) & 1, z = (zw >> b) & 1;
      if (x && z) extra += 3;
      if (x) {
        const uint64_t* cr = c + (uint64_t)q * W;
#pragma unroll
        for (int k = 0; k < PER; k++) {
          const uint32_t w = lane + 32 * k;
          if (w < len) mul_step<uint64_t>(__ldg(cr + w), __ldg(cr + len + w), bx[k], bz[k], c1[k], c2[k]);
        }
        extra += cph[q];
      }
      if (z) {
        const uint64_t* cr = c + (uint64_t)(q + n) * W;
#pragma unroll
        for (int k = 0; k < PER; k++) {
          const uint32_t w = lane + 32 * k;
          if (w < len) mul_step<uint64_t>(__ldg(cr + w), __ldg(cr + len + w), bx[k], bz[k], c1[k], c2[k]);
        }
        extra += cph[q + n];
      }
    }
  }
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < PER; k++) s += cnt_phase(c1[k], c2[k]);
  s = __reduce_add_sync(0xFFFFFFFFu, s & 3u) & 3u;
#pragma unroll
  for (int k = 0; k < PER; k++) {
    const uint32_t w = lane + 32 * k;
    if (w < len) { part[g][w] = bx[k]; part[g][len + w] = bz[k]; }
  }
  if (lane == 0) pph[g] = (s + extra) & 3u;
  __syncthreads();
  if (g != 0) return;
  // warp 0: acc = P_0, then acc <- P_g * acc for g = 1 .. G-1
#pragma unroll
  for (int k = 0; k < PER; k++) { c1[k] = c2[k] = 0; }
  uint32_t tot = pph[0];
  for (uint32_t h = 1; h < G; h++) {
#pragma unroll
    for (int k = 0; k < PER; k++) {
      const uint32_t w = lane + 32 * k;
      if (w < len) mul_step<uint64_t>(part[h][w], part[h][len + w], bx[k], bz[k], c1[k], c2[k]);
    }
    tot += pph[h];
  }
  s = 0;
#pragma unroll
  for (int k = 0; k < PER; k++) s += cnt_phase(c1[k], c2[k]);
  s = __reduce_add_sync(0xFFFFFFFFu, s & 3u) & 3u;
#pragma unroll
  for (int k = 0; k < PER; k++) {
    const uint32_t w = lane + 32 * k;
    if (w < len) { row[w] = bx[k]; row[len + w] = bz[k]; }
  }
  if (lane == 0) ph[r] = phases ? (uint8_t)((s + tot + ph[r]) & 3u) : (uint8_t)0;
}

// rowswap!(state, i, j; phases) (src/QuantumClifford.jl:899-927): rows i and
// j of the view (and their destabilizer rows for the Destabilizer kinds), the
// phases only when `phases`.  One thread per word.
__global__ void rowswap_kernel(uint64_t* xzs, uint8_t* ph, uint32_t W, uint32_t i, uint32_t j, uint32_t di,
                               uint32_t dj, int destab, int phases) {
  const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w < W) {
    uint64_t t = xzs[(size_t)i * W + w]; xzs[(size_t)i * W + w] = xzs[(size_t)j * W + w]; xzs[(size_t)j * W + w] = t;
    if (destab) { t = xzs[(size_t)di * W + w]; xzs[(size_t)di * W + w] = xzs[(size_t)dj * W + w]; xzs[(size_t)dj * W + w] = t; }
  }
  if (w == 0 && phases) {
    uint8_t p = ph[i]; ph[i] = ph[j]; ph[j] = p;
    if (destab) { p = ph[di]; ph[di] = ph[dj]; ph[dj] = p; }
  }
}

// ---------------------------------------------------------------- no-alloc batch
// Phase accumulators of qcb_mul_left_pauli_batch_noalloc, one per pair.  Zero
// between calls: the finish kernel clears what it read.
static __device__ __align__(256) uint32_t g_noalloc_acc[QCB_NOALLOC_MAX_PAIRS];

// Pair blockIdx.y of a batch: the grid-stride loop of mul_left_long_kernel
// over that pair's words, the phase sum added into acc[pair].
template <int VEC, bool PH>
__global__ void __launch_bounds__(256) mul_left_batch_kernel(uint64_t* __restrict__ r,
                                                             const uint64_t* __restrict__ l,
                                                             uint64_t len, uint32_t* acc) {
  const uint32_t pair = blockIdx.y;
  r += (uint64_t)pair * 2 * len;
  l += (uint64_t)pair * 2 * len;
  uint64_t c1a = 0, c2a = 0, c1b = 0, c2b = 0;
  const uint64_t nvec = len / VEC;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nvec; i += stride) {
    if (VEC == 2) {
      const ulonglong2 lx = __ldcs((const ulonglong2*)l + i);
      const ulonglong2 lz = __ldcs((const ulonglong2*)(l + len) + i);
      ulonglong2 rx = __ldcs((const ulonglong2*)r + i);
      ulonglong2 rz = __ldcs((const ulonglong2*)(r + len) + i);
      if (PH) {
        mul_step(lx.x, lz.x, rx.x, rz.x, c1a, c2a);
        mul_step(lx.y, lz.y, rx.y, rz.y, c1b, c2b);
      } else {
        rx.x ^= lx.x; rx.y ^= lx.y; rz.x ^= lz.x; rz.y ^= lz.y;
      }
      __stcs((ulonglong2*)r + i, rx);
      __stcs((ulonglong2*)(r + len) + i, rz);
    } else {
      const uint64_t lx = __ldcs(l + i), lz = __ldcs(l + len + i);
      uint64_t rx = __ldcs(r + i), rz = __ldcs(r + len + i);
      if (PH) mul_step(lx, lz, rx, rz, c1a, c2a);
      else { rx ^= lx; rz ^= lz; }
      __stcs(r + i, rx);
      __stcs(r + len + i, rz);
    }
  }
  if (!PH) return;
  uint32_t v = (cnt_phase(c1a, c2a) + cnt_phase(c1b, c2b)) & 3u;
  v = __reduce_add_sync(0xFFFFFFFFu, v) & 3u;
  __shared__ uint32_t wsum[32];
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) wsum[wid] = v;
  __syncthreads();
  if (wid == 0) {
    uint32_t s = lane < (blockDim.x >> 5) ? wsum[lane] : 0u;
    s = __reduce_add_sync(0xFFFFFFFFu, s) & 3u;
    if (lane == 0 && s) atomicAdd(acc + pair, s);
  }
}

// r_phase[i] <- (s_i + r_phase[i] + l_phase[i]) & 3 (src/mul_leftright.jl:140)
// when phases; clears acc[i] either way.
__global__ void mul_left_batch_finish_kernel(uint8_t* r_phase, const uint8_t* l_phase, uint32_t* acc,
                                             uint32_t count, int phases) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  if (phases) r_phase[i] = (uint8_t)(((acc[i] & 3u) + r_phase[i] + l_phase[i]) & 3u);
  acc[i] = 0;
}

static uint32_t g_gates_pdl = 1;  // symbolic gate launches as programmatic dependents (0: plain)
void set_gates_pdl(uint32_t v) { g_gates_pdl = v; }

}  // namespace qcb

using namespace qcb;

extern "C" {

int qcb_mul_left_pauli(qcb_tableau* r, const qcb_tableau* l, int phases, uint8_t* phase_out,
                       void* stream) {
  if (!r || !l) return fail(QCB_EARG, "null argument");
  if (r->nqubits != l->nqubits)
    return fail(QCB_EDIM, "The two Pauli operators should have the same length!");
  if (r->rows < 1 || l->rows < 1) return fail(QCB_EDIM, "empty Pauli");
  const uint64_t len = r->W / 2;
  cudaStream_t st = S(stream);
  const int sms = device_sm_count();
  const bool vec = (len % 2 == 0);
  const uint64_t work = vec ? len / 2 : len;
  // one wave of resident blocks (no tail wave for the grid-stride loop)
  void (*k)(uint64_t*, const uint64_t*, uint64_t, uint32_t*, uint8_t*, const uint8_t*) =
      vec ? (phases ? mul_left_long_kernel<2, true> : mul_left_long_kernel<2, false>)
          : (phases ? mul_left_long_kernel<1, true> : mul_left_long_kernel<1, false>);
  int per_sm = 0;
  QCB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 256, 0));
  uint32_t blocks = (uint32_t)std::min<uint64_t>((work + 255) / 256, (uint64_t)sms * std::max(per_sm, 1));
  if (blocks == 0) blocks = 1;
  if (len) {
    k<<<blocks, 256, 0, st>>>(r->xzs, l->xzs, len, r->scratch, r->phases, l->phases);
    QCB_LAUNCHED();
  } else if (phases) {
    mul_left_finish_kernel<<<1, 1, 0, st>>>(r->phases, l->phases, r->scratch, phases);
    QCB_LAUNCHED();
  }
  if (phase_out) {
    QCB_CUDA(cudaMemcpyAsync(phase_out, r->phases, 1, cudaMemcpyDeviceToHost, st));
    QCB_CUDA(cudaStreamSynchronize(st));
  }
  return QCB_OK;
}

int qcb_rowswap(qcb_tableau* t, int kind, uint32_t i, uint32_t j, int phases, void* stream) {
  if (!t) return fail(QCB_EARG, "null tableau");
  if (i == 0 || j == 0) return fail(QCB_EBOUNDS, "rows are 1-based");
  const bool destab = kind == QCB_DESTABILIZER || kind == QCB_MIXED_DESTABILIZER;
  if (kind < 0 || kind > 3) return fail(QCB_EARG, "rowswap!: bad state kind");
  if (destab && t->rows % 2) return fail(QCB_EDIM, "destabilizer tableaux have an even number of rows");
  const uint32_t nn = destab ? t->rows / 2 : t->rows;
  if (i > nn || j > nn) return fail(QCB_EBOUNDS, "rowswap!: row out of range");
  if (i == j) return QCB_OK;
  const uint32_t off = destab ? nn : 0;
  rowswap_kernel<<<(t->W + 127) / 128, 128, 0, S(stream)>>>(t->xzs, t->phases, t->W, off + i - 1, off + j - 1, i - 1,
                                                           j - 1, destab ? 1 : 0, phases);
  QCB_LAUNCHED();
  return QCB_OK;
}

int qcb_mul_rows(qcb_tableau* s, uint32_t s_row, uint32_t count, const qcb_tableau* t, uint32_t t_row,
                 uint32_t t_step, int right, int phase_src, int phases, uint8_t* phase_out, void* stream) {
  if (!s || !t) return fail(QCB_EARG, "null tableau");
  if (s->nqubits != t->nqubits) return fail(QCB_EDIM, "The two Pauli operators should have the same length!");
  if (!count) return QCB_OK;
  const uint64_t last_b = (uint64_t)t_row + (uint64_t)(count - 1) * t_step;
  if (s_row < 1 || t_row < 1 || (uint64_t)s_row + count - 1 > s->rows || last_b > t->rows)
    return fail(QCB_EBOUNDS, "row index out of bounds");
  if (phase_src && last_b > s->rows) return fail(QCB_EBOUNDS, "row index out of bounds (phase taken from s)");
  if (s == t && count > 1) {  // rows read by one warp must not be written by another
    const bool same = (t_row == s_row && t_step == 1);
    const uint64_t b_lo = t_row, b_hi = last_b;
    const bool disjoint = (b_hi < s_row || b_lo >= (uint64_t)s_row + count);
    if (!same && !disjoint)
      return fail(QCB_EARG, "source rows overlap the target rows of the same tableau");
  }
  cudaStream_t st = S(stream);
  const uint8_t* add = phase_src ? s->phases : t->phases;
  const uint32_t a0 = s_row - 1, b0 = t_row - 1;
  const uint64_t len = s->W / 2;
  if (count == 1 && len >= (1u << 15)) {
    // one long row: the grid-stride kernel of mul_left!(::PauliOperator, ...)
    const bool vec = (len % 2 == 0);
    uint64_t* r = s->xzs + (uint64_t)a0 * s->W;
    const uint64_t* l = t->xzs + (uint64_t)b0 * t->W;
    const bool aligned = ((uintptr_t)r % 16 == 0) && ((uintptr_t)l % 16 == 0);
    void (*k)(uint64_t*, const uint64_t*, uint64_t, uint32_t*, uint8_t*, const uint8_t*);
    if (vec && aligned)
      k = right ? (phases ? mul_left_long_kernel<2, true, true> : mul_left_long_kernel<2, false, true>)
                : (phases ? mul_left_long_kernel<2, true> : mul_left_long_kernel<2, false>);
    else
      k = right ? (phases ? mul_left_long_kernel<1, true, true> : mul_left_long_kernel<1, false, true>)
                : (phases ? mul_left_long_kernel<1, true> : mul_left_long_kernel<1, false>);
    int per_sm = 0;
    QCB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 256, 0));
    const uint64_t work = (vec && aligned) ? len / 2 : len;
    uint32_t blocks = (uint32_t)std::min<uint64_t>((work + 255) / 256,
                                                   (uint64_t)device_sm_count() * std::max(per_sm, 1));
    k<<<std::max(blocks, 1u), 256, 0, st>>>(r, l, len, s->scratch, s->phases + a0, add + b0);
    QCB_LAUNCHED();
  } else {
    const uint32_t warps_per_block = 8;
    const uint32_t blocks = (uint32_t)std::min<uint64_t>((count + warps_per_block - 1) / warps_per_block,
                                                         (uint64_t)device_sm_count() * 16);
    void (*k)(uint64_t*, uint8_t*, uint32_t, uint32_t, const uint64_t*, uint32_t, uint32_t, uint32_t,
              const uint8_t*) = right ? (phases ? mul_rows_kernel<true, true> : mul_rows_kernel<true, false>)
                                      : (phases ? mul_rows_kernel<false, true> : mul_rows_kernel<false, false>);
    k<<<blocks, 256, 0, st>>>(s->xzs, s->phases, a0, count, t->xzs, b0, t_step, s->W, add);
    QCB_LAUNCHED();
  }
  if (phase_out) {
    QCB_CUDA(cudaMemcpyAsync(phase_out, s->phases + a0, 1, cudaMemcpyDeviceToHost, st));
    QCB_CUDA(cudaStreamSynchronize(st));
  }
  return QCB_OK;
}

int qcb_mul_left_state(qcb_tableau* s, int kind, uint32_t i, uint32_t j, int phases, void* stream) {
  if (!s) return fail(QCB_EARG, "null tableau");
  if (kind == QCB_DESTABILIZER || kind == QCB_MIXED_DESTABILIZER) {
    // src/mul_leftright.jl:200-219: destabilizer j <- destabilizer i * j
    // without phases (indices flipped), then stabilizer i <- stabilizer j * i
    if (s->rows % 2) return fail(QCB_EDIM, "a Destabilizer tableau has 2n rows");
    const uint32_t n = s->rows / 2;
    if (i < 1 || j < 1 || i > n || j > n) return fail(QCB_EBOUNDS, "row index out of bounds");
    if (int st = qcb_mul_rows(s, j, 1, s, i, 0, 0, 0, 0, nullptr, stream)) return st;
    return qcb_mul_rows(s, i + n, 1, s, j + n, 0, 0, 0, phases, nullptr, stream);
  }
  if (kind != QCB_STABILIZER && kind != QCB_MIXED_STABILIZER) return fail(QCB_EARG, "unknown state kind");
  // src/mul_leftright.jl:194-198, 207-211: rows of the tableau
  return qcb_mul_rows(s, i, 1, s, j, 0, 0, 0, phases, nullptr, stream);
}

int qcb_mul_left_row(qcb_tableau* s, uint32_t m, uint32_t i, int phases, void* stream) {
  if (!s) return fail(QCB_EARG, "null tableau");
  if (m < 1 || i < 1 || m > s->rows || i > s->rows) return fail(QCB_EBOUNDS, "row index out of bounds");
  mul_left_row_kernel<<<1, 32, 0, S(stream)>>>(s->xzs, s->phases, s->W, m - 1, i - 1, phases);
  QCB_LAUNCHED();
  return QCB_OK;
}

int qcb_mul_left_tableau_pauli(qcb_tableau* s, const qcb_tableau* p, int phases, void* stream) {
  if (!s || !p) return fail(QCB_EARG, "null argument");
  if (s->nqubits != p->nqubits) return fail(QCB_EDIM, "The tableau and the Pauli operator must have the same number of qubits");
  if (!s->rows) return QCB_OK;
  const uint32_t threads = 256, blocks = (s->rows * 32 + threads - 1) / threads;
  mul_left_tab_pauli_kernel<<<blocks, threads, 0, S(stream)>>>(s->xzs, s->phases, s->rows, s->W,
                                                               p->xzs, p->phases, phases);
  QCB_LAUNCHED();
  return QCB_OK;
}

static int pc_common(const qcb_tableau* l, uint32_t i, const qcb_tableau* r, uint32_t j, uint8_t* out,
                     void* stream, int what) {
  if (!l || !r || !out) return fail(QCB_EARG, "null argument");
  if (l->nqubits != r->nqubits) return fail(QCB_EDIM, "operands must have the same number of qubits");
  if (i < 1 || i > l->rows || j < 1 || j > r->rows) return fail(QCB_EBOUNDS, "row index out of bounds");
  cudaStream_t st = S(stream);
  uint8_t lph = 0, rph = 0;
  QCB_CUDA(cudaMemcpyAsync(&lph, l->phases + (i - 1), 1, cudaMemcpyDeviceToHost, st));
  QCB_CUDA(cudaMemcpyAsync(&rph, r->phases + (j - 1), 1, cudaMemcpyDeviceToHost, st));
  QCB_CUDA(cudaStreamSynchronize(st));
  uint8_t* d = (uint8_t*)l->scratch + 64;
  prodphase_comm_kernel<<<1, 32, 0, st>>>(l->xzs + (uint64_t)(i - 1) * l->W, lph,
                                          r->xzs + (uint64_t)(j - 1) * r->W, rph, l->W / 2, what, d);
  QCB_LAUNCHED();
  QCB_CUDA(cudaMemcpyAsync(out, d, 1, cudaMemcpyDeviceToHost, st));
  QCB_CUDA(cudaStreamSynchronize(st));
  return QCB_OK;
}

int qcb_prodphase(const qcb_tableau* l, uint32_t i, const qcb_tableau* r, uint32_t j, uint8_t* out,
                  void* stream) {
  return pc_common(l, i, r, j, out, stream, 0);
}

int qcb_comm(const qcb_tableau* l, uint32_t i, const qcb_tableau* r, uint32_t j, uint8_t* out,
             void* stream) {
  return pc_common(l, i, r, j, out, stream, 1);
}

int qcb_apply_gates(qcb_tableau* t, const qcb_op* ops, size_t n_ops, int phases, void* stream) {
  if (!t) return fail(QCB_EARG, "null tableau");
  std::vector<GateOp> g;
  g.reserve(n_ops);
  for (size_t k = 0; k < n_ops; k++) {
    const qcb_op& o = ops[k];
    const bool one = o.opcode >= QCB_OP_I && o.opcode <= QCB_OP_SQO;
    const bool two = o.opcode >= QCB_OP_CNOT && o.opcode <= QCB_OP_LAST2Q;
    if (!one && !two) return fail(QCB_EUNSUPPORTED, "qcb_apply_gates: op " + std::to_string(k) + " is not a symbolic Clifford gate");
    if (o.q1 == 0 || (two && o.q2 == 0)) return fail(QCB_EZEROQUBIT, "qubit indices start at 1 (NoZeroQubit)");
    if (two && o.q1 == o.q2) return fail(QCB_EARG, "Failed to create a two qubit gate because the two qubits it acts on have the same index. The qubit indices have to be different.");
    if (o.q1 > t->nqubits || (two && o.q2 > t->nqubits)) return fail(QCB_EBOUNDS, "gate qubit index exceeds the tableau's qubits");
    const uint32_t code = o.opcode == QCB_OP_SQO ? o.opcode | ((o.q2 & 63u) << 8) : o.opcode;
    g.push_back({code, o.q1 - 1, two ? o.q2 - 1 : 0, 0});
  }
  if (g.empty() || !t->rows) return QCB_OK;
  cudaStream_t st = S(stream);
  for (size_t k0 = 0; k0 < g.size(); k0 += GATE_BATCH) {
    const uint32_t n = (uint32_t)std::min<size_t>(GATE_BATCH, g.size() - k0);
    GateBatch b{};
    std::copy(g.begin() + k0, g.begin() + k0 + n, b.op);
    // a programmatic dependent of the previous launch on the stream: in a
    // stream of single-gate calls each launch is scheduled while the one
    // before it runs, instead of after it drains
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((t->rows + 127) / 128);
    cfg.blockDim = dim3(128);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = g_gates_pdl ? 1 : 0;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    QCB_CUDA(cudaLaunchKernelEx(&cfg, apply_gates_kernel, t->xzs, t->phases, t->rows, t->W, (const GateBatch)b, n, phases));
    QCB_LAUNCHED();
  }
  return QCB_OK;
}

int qcb_apply_dense(qcb_tableau* t, const qcb_tableau* c, int phases, void* stream) {
  if (!t || !c) return fail(QCB_EARG, "null argument");
  if (t->nqubits != c->nqubits || c->rows != 2 * c->nqubits)
    return fail(QCB_EDIM, "The tableau and the Clifford operator need to act on the same number of qubits.");
  if (!t->rows) return QCB_OK;
  cudaStream_t st = S(stream);
  const uint32_t W = t->W;
  // 8 warps per row (one row per CTA) unless the rows alone fill the GPU
  const bool split = (uint64_t)t->rows < 8ull * 148 * 8 && W >= 16;
  if (split) {
    if (W <= 64)
      apply_dense_split_kernel<64, 8><<<t->rows, 256, 0, st>>>(t->xzs, t->phases, t->rows, W, t->nqubits, c->xzs, c->phases, phases);
    else if (W <= 128)
      apply_dense_split_kernel<128, 8><<<t->rows, 256, 0, st>>>(t->xzs, t->phases, t->rows, W, t->nqubits, c->xzs, c->phases, phases);
    else if (W <= 256)
      apply_dense_split_kernel<256, 8><<<t->rows, 256, 0, st>>>(t->xzs, t->phases, t->rows, W, t->nqubits, c->xzs, c->phases, phases);
    else
      return fail(QCB_EUNSUPPORTED, "qcb_apply_dense: at most 8192 qubits");
    QCB_LAUNCHED();
    return QCB_OK;
  }
  const uint32_t threads = 256, blocks = (t->rows * 32 + threads - 1) / threads;
  if (W <= 64)
    apply_dense_kernel<64><<<blocks, threads, 0, st>>>(t->xzs, t->phases, t->rows, W, t->nqubits, c->xzs, c->phases, phases);
  else if (W <= 128)
    apply_dense_kernel<128><<<blocks, threads, 0, st>>>(t->xzs, t->phases, t->rows, W, t->nqubits, c->xzs, c->phases, phases);
  else if (W <= 256)
    apply_dense_kernel<256><<<blocks, threads, 0, st>>>(t->xzs, t->phases, t->rows, W, t->nqubits, c->xzs, c->phases, phases);
  else
    return fail(QCB_EUNSUPPORTED, "qcb_apply_dense: at most 8192 qubits");
  QCB_LAUNCHED();
  return QCB_OK;
}

// The no-alloc scratch of the current device: looked up once per device with
// that device current, cleared once, then reused by every call.
static std::mutex g_noalloc_mu;
static uint32_t* g_noalloc_ptr[64] = {};

static int noalloc_scratch(uint32_t** out) {
  int dev = 0;
  QCB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(QCB_EARG, "device ordinal out of range for the no-alloc scratch");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    uint32_t* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_acc);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
    e = cudaMemset(p, 0, sizeof(uint32_t) * QCB_NOALLOC_MAX_PAIRS);
    if (e != cudaSuccess) return cuda_fail(e, "clearing the no-alloc scratch");
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(e, "clearing the no-alloc scratch");
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return QCB_OK;
}

int qcb_mul_left_pauli_batch_noalloc(uint64_t* r_xz, uint8_t* r_phases, const uint64_t* l_xz,
                                     const uint8_t* l_phases, uint32_t nqubits, uint32_t count,
                                     int phases, void* stream) {
  if (count == 0) return QCB_OK;
  if (count > QCB_NOALLOC_MAX_PAIRS)
    return fail(QCB_EARG, "qcb_mul_left_pauli_batch_noalloc: count " + std::to_string(count) +
                              " exceeds the no-alloc scratch of " + std::to_string(QCB_NOALLOC_MAX_PAIRS) +
                              " pairs; split the batch");
  if (!r_xz || !l_xz) return fail(QCB_EARG, "qcb_mul_left_pauli_batch_noalloc: null Pauli words");
  if (phases && (!r_phases || !l_phases)) return fail(QCB_EARG, "qcb_mul_left_pauli_batch_noalloc: null phases");
  uint32_t* acc = nullptr;
  if (int st = noalloc_scratch(&acc)) return st;
  const uint64_t len = ((uint64_t)nqubits + 63) / 64;
  cudaStream_t st = S(stream);
  const bool vec = len % 2 == 0 && (((uintptr_t)r_xz | (uintptr_t)l_xz) & 15u) == 0;
  const uint64_t work = vec ? len / 2 : len;
  const uint32_t bx = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((work + 255) / 256, (uint64_t)device_sm_count() * 8));
  if (len) {
    const dim3 grid(bx, count);
    if (vec) {
      if (phases) mul_left_batch_kernel<2, true><<<grid, 256, 0, st>>>(r_xz, l_xz, len, acc);
      else mul_left_batch_kernel<2, false><<<grid, 256, 0, st>>>(r_xz, l_xz, len, acc);
    } else {
      if (phases) mul_left_batch_kernel<1, true><<<grid, 256, 0, st>>>(r_xz, l_xz, len, acc);
      else mul_left_batch_kernel<1, false><<<grid, 256, 0, st>>>(r_xz, l_xz, len, acc);
    }
    QCB_LAUNCHED();
  }
  mul_left_batch_finish_kernel<<<(count + 255) / 256, 256, 0, st>>>(r_phases, l_phases, acc, count, phases);
  QCB_LAUNCHED();
  return QCB_OK;
}

}  // extern "C"
