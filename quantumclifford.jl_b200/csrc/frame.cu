// frame.cu -- Pauli-frame engine: frame storage, the whole-circuit walker
// kernel, noise sources and reference-layout transposes.
//
// Reference path replaced: PauliFrame / initZ! / apply!(::PauliFrame, ...) /
// applynoise! / pftrajectories (src/pauli_frames.jl:9-257) and the CUDA
// extension's per-op kernels (ext/QuantumCliffordGPUExt/apply.jl:7-136,
// pauli_frames.jl:7-60, apply_noise.jl:5-38).
//
// Layout.  A frame of S shots over nq1 = qubits+1 qubits is stored as bit
// planes packed along shots: plane 2q holds the x bits of qubit q, plane 2q+1
// its z bits, one uint32 word per 32 shots ("column").  The record is one
// plane per measurement bit.  A column is independent of every other column
// under every frame operation, so one thread owns one column for the whole
// circuit: it walks the compiled program, keeping its column of every touched
// qubit in shared memory (or in the HBM planes when the frame is too tall),
// and only the record and the final frame go to HBM.
//
// Noise (Philox mode).  Each column draws its own counter-based stream
// (key = seed, counter = (draw, column, tag)).  Noise sites are visited in
// program order; over the trials t = site*32 + lane the column samples the
// gaps between events geometrically at rate p_max, then picks the event kind
// (or thins it away) from a second uniform scaled by p_max.  Events of sites
// [b, e) are applied at the FLUSH record the compiler placed for them.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <unordered_map>

#include "qcb_internal.h"

namespace qcb {

struct WalkArgs {
  const uint4* prog;
  uint32_t* planes;
  uint32_t* rec;
  uint64_t pitch;
  uint64_t ncols;
  const uint32_t* slot_qubit;
  uint32_t nslots;
  uint32_t scratch_plane;  // qubit index of the scratch plane pair
  uint32_t nq1;
  uint32_t fresh;          // 1: start from x = 0, z = Philox initZ!
  const uint32_t* qubit_slot;
  uint32_t qubit_slot_len;
  uint32_t nsites;
  uint64_t seed;
  uint64_t col0;           // global column index of column 0
  const Site* sites;
  double pmax;
  double inv_log1m;
  // mask mode
  const uint64_t* ev_off;
  const uint64_t* ev_data;  // (trial << 8) | code, sorted per column
  const uint32_t* reset_planes;
  uint64_t reset_pitch;
};

// Column storage: shared memory tile or HBM planes.
struct SmemCol {
  uint32_t* b;   // sm + tid
  uint32_t nt;
  __device__ __forceinline__ uint32_t& x(uint32_t s) const { return b[(2 * s) * nt]; }
  __device__ __forceinline__ uint32_t& z(uint32_t s) const { return b[(2 * s + 1) * nt]; }
};
struct GlobCol {
  uint32_t* b;   // planes + c
  const uint32_t* po;  // slot -> plane pair (shared memory table)
  uint64_t p;
  __device__ __forceinline__ uint32_t& x(uint32_t s) const { return b[(uint64_t)(2 * po[s]) * p]; }
  __device__ __forceinline__ uint32_t& z(uint32_t s) const { return b[(uint64_t)(2 * po[s] + 1) * p]; }
};

__device__ __forceinline__ uint32_t sel4(const uint32_t o[4], uint32_t i) {
  uint32_t a = (i & 1) ? o[1] : o[0];
  uint32_t b = (i & 1) ? o[3] : o[2];
  return (i & 2) ? b : a;
}

struct NoiseState {
  uint64_t t;
  double v;
  uint32_t draw;
  bool alive;
};

__device__ __forceinline__ void noise_step(NoiseState& ns, const WalkArgs& a, uint64_t col,
                                           bool first) {
  uint32_t o[4];
  philox4x32_10(ns.draw++, (uint32_t)col, (uint32_t)(col >> 32), TAG_NOISE, (uint32_t)a.seed,
                (uint32_t)(a.seed >> 32), o);
  uint64_t u53 = ((uint64_t)o[0] << 21) | (o[1] >> 11);
  double u = __dmul_rn(__dadd_rn((double)u53, 0.5), 0x1.0p-53);
  double g = a.pmax >= 1.0 ? 0.0 : floor(__dmul_rn(log(u), a.inv_log1m));
  ns.v = __dmul_rn(__dmul_rn((double)o[2], 0x1.0p-32), a.pmax);
  if (g > 9.0e18) {
    ns.alive = false;
    return;
  }
  uint64_t gi = (uint64_t)g;
  ns.t = first ? gi : ns.t + 1 + gi;
}

__device__ __forceinline__ uint32_t site_code(const Site& s, double v) {
  if (s.kind == QCB_OP_PAULI_NOISE) {
    if (v < s.t0) return 1;
    if (v < s.t1) return 2;
    if (v < s.t2) return 3;
    return 0;
  }
  uint32_t np = s.kind == QCB_OP_DEPOL2 ? 15u : 3u;
  if (v < s.t0) {
    uint32_t k = (uint32_t)(__dmul_rn(v / s.t0, (double)np));
    if (k >= np) k = np - 1;
    return k + 1;
  }
  return 0;
}

template <class Col>
__device__ __forceinline__ void flip(const Col& C, uint32_t s, uint32_t digit, uint32_t bit) {
  if (digit & 1) C.x(s) ^= bit;
  if (digit & 2) C.z(s) ^= bit;
}

template <class Col>
__device__ __forceinline__ void apply_event(const Col& C, const Site& s, uint32_t code,
                                            uint32_t bit) {
  if (s.kind == QCB_OP_DEPOL2) {
    flip(C, s.a, code & 3, bit);
    flip(C, s.b, (code >> 2) & 3, bit);
  } else {
    flip(C, s.a, code & 3, bit);
  }
}

// Bit-sliced single-qubit gate (src/symbolic_cliffords.jl:105-118), frames
// track no phase (src/pauli_frames.jl:58-61).
__device__ __forceinline__ void gate1_xz(uint32_t op, uint32_t& x, uint32_t& z) {
  uint32_t X = x, Z = z;
  switch (op) {
    case QCB_OP_H: case QCB_OP_SQRTY: case QCB_OP_INVSQRTY: x = Z; z = X; break;
    case QCB_OP_HXY: case QCB_OP_S: case QCB_OP_SDAG: x = X; z = X ^ Z; break;
    case QCB_OP_HYZ: case QCB_OP_SQRTX: case QCB_OP_INVSQRTX: x = X ^ Z; z = Z; break;
    case QCB_OP_CXYZ: x = X ^ Z; z = X; break;
    case QCB_OP_CZYX: x = Z; z = X ^ Z; break;
    default: break;  // I, X, Y, Z: no change to the frame bits
  }
}

// Bit-sliced two-qubit gate maps (src/symbolic_cliffords.jl:358-395).
__device__ __forceinline__ void gate2_xz(uint32_t op, uint32_t& x1, uint32_t& z1, uint32_t& x2,
                                         uint32_t& z2) {
  uint32_t a = x1, b = z1, c = x2, d = z2;
  switch (op) {
    case QCB_OP_SWAP: x1 = c; z1 = d; x2 = a; z2 = b; break;
    case QCB_OP_CNOT: case QCB_OP_ZCX: z1 = b ^ d; x2 = c ^ a; break;
    case QCB_OP_CPHASE: case QCB_OP_ZCZ: z1 = b ^ c; z2 = d ^ a; break;
    case QCB_OP_ZCY: z1 = c ^ b ^ d; x2 = c ^ a; z2 = d ^ a; break;
    case QCB_OP_XCX: x1 = d ^ a; x2 = c ^ b; break;
    case QCB_OP_XCY: x1 = a ^ c ^ d; x2 = b ^ c; z2 = d ^ b; break;
    case QCB_OP_XCZ: x1 = a ^ c; z2 = d ^ b; break;
    case QCB_OP_YCX: x1 = a ^ d; z1 = d ^ b; x2 = a ^ b ^ c; break;
    case QCB_OP_YCY: x1 = a ^ d ^ c; z1 = b ^ c ^ d; x2 = a ^ c ^ b; z2 = a ^ b ^ d; break;
    case QCB_OP_YCZ: x1 = a ^ c; z1 = c ^ b; z2 = d ^ a ^ b; break;
    default: break;
  }
}

template <class Col, bool PHILOX>
__device__ __forceinline__ void walk_column(const WalkArgs& a, const Col& C, uint64_t c) {
  const uint64_t col = a.col0 + c;
  const uint32_t k0 = (uint32_t)a.seed, k1 = (uint32_t)(a.seed >> 32);
  const uint32_t clo = (uint32_t)col, chi = (uint32_t)(col >> 32);
  uint32_t* rec = a.rec + c;
  const uint64_t pitch = a.pitch;

  NoiseState ns{0, 0.0, 0, false};
  uint64_t ep = 0, ee = 0;
  if (PHILOX) {
    if (a.nsites && a.pmax > 0.0) {
      ns.alive = true;
      noise_step(ns, a, col, true);
    }
  } else {
    ep = a.ev_off[c];
    ee = a.ev_off[c + 1];
  }
  uint32_t rblk = 0xFFFFFFFFu;
  uint32_t rc[4] = {0, 0, 0, 0};

  const uint4* pc = a.prog;
  while (true) {
    const uint4 h = __ldg(pc++);
    const uint32_t kind = h.x >> 24, cnt = h.x & 0xFFFFFFu;
    if (kind == SEG_END) break;
    switch (kind) {
      case SEG_CNOT: {
        for (uint32_t i = 0; i < cnt; i += 4) {
          const uint4 o0 = __ldg(pc), o1 = __ldg(pc + 1);
          pc += 2;
          uint32_t xc0 = C.x(o0.x), zc0 = C.z(o0.x), xt0 = C.x(o0.y), zt0 = C.z(o0.y);
          uint32_t xc1 = C.x(o0.z), zc1 = C.z(o0.z), xt1 = C.x(o0.w), zt1 = C.z(o0.w);
          uint32_t xc2 = C.x(o1.x), zc2 = C.z(o1.x), xt2 = C.x(o1.y), zt2 = C.z(o1.y);
          uint32_t xc3 = C.x(o1.z), zc3 = C.z(o1.z), xt3 = C.x(o1.w), zt3 = C.z(o1.w);
          C.x(o0.y) = xt0 ^ xc0; C.z(o0.x) = zc0 ^ zt0;
          C.x(o0.w) = xt1 ^ xc1; C.z(o0.z) = zc1 ^ zt1;
          C.x(o1.y) = xt2 ^ xc2; C.z(o1.x) = zc2 ^ zt2;
          C.x(o1.w) = xt3 ^ xc3; C.z(o1.z) = zc3 ^ zt3;
        }
        break;
      }
      case SEG_CZ: {
        for (uint32_t i = 0; i < cnt; i += 4) {
          const uint4 o0 = __ldg(pc), o1 = __ldg(pc + 1);
          pc += 2;
          uint32_t xa0 = C.x(o0.x), za0 = C.z(o0.x), xb0 = C.x(o0.y), zb0 = C.z(o0.y);
          uint32_t xa1 = C.x(o0.z), za1 = C.z(o0.z), xb1 = C.x(o0.w), zb1 = C.z(o0.w);
          uint32_t xa2 = C.x(o1.x), za2 = C.z(o1.x), xb2 = C.x(o1.y), zb2 = C.z(o1.y);
          uint32_t xa3 = C.x(o1.z), za3 = C.z(o1.z), xb3 = C.x(o1.w), zb3 = C.z(o1.w);
          C.z(o0.x) = za0 ^ xb0; C.z(o0.y) = zb0 ^ xa0;
          C.z(o0.z) = za1 ^ xb1; C.z(o0.w) = zb1 ^ xa1;
          C.z(o1.x) = za2 ^ xb2; C.z(o1.y) = zb2 ^ xa2;
          C.z(o1.z) = za3 ^ xb3; C.z(o1.w) = zb3 ^ xa3;
        }
        break;
      }
      case SEG_H: {
        for (uint32_t i = 0; i < cnt; i += 4) {
          const uint4 o = __ldg(pc++);
          uint32_t x0 = C.x(o.x), z0 = C.z(o.x), x1 = C.x(o.y), z1 = C.z(o.y);
          uint32_t x2 = C.x(o.z), z2 = C.z(o.z), x3 = C.x(o.w), z3 = C.z(o.w);
          C.x(o.x) = z0; C.z(o.x) = x0; C.x(o.y) = z1; C.z(o.y) = x1;
          C.x(o.z) = z2; C.z(o.z) = x2; C.x(o.w) = z3; C.z(o.w) = x3;
        }
        break;
      }
      case SEG_S: {
        for (uint32_t i = 0; i < cnt; i += 4) {
          const uint4 o = __ldg(pc++);
          uint32_t x0 = C.x(o.x), z0 = C.z(o.x), x1 = C.x(o.y), z1 = C.z(o.y);
          uint32_t x2 = C.x(o.z), z2 = C.z(o.z), x3 = C.x(o.w), z3 = C.z(o.w);
          C.z(o.x) = z0 ^ x0; C.z(o.y) = z1 ^ x1; C.z(o.z) = z2 ^ x2; C.z(o.w) = z3 ^ x3;
        }
        break;
      }
      case SEG_G1: {
        for (uint32_t i = 0; i < cnt; i += 2) {
          const uint4 o = __ldg(pc++);
          uint32_t x0 = C.x(o.y), z0 = C.z(o.y), x1 = C.x(o.w), z1 = C.z(o.w);
          gate1_xz(o.x, x0, z0);
          gate1_xz(o.z, x1, z1);
          C.x(o.y) = x0; C.z(o.y) = z0; C.x(o.w) = x1; C.z(o.w) = z1;
        }
        break;
      }
      case SEG_G2: {
        for (uint32_t i = 0; i < cnt; i++) {
          const uint4 o = __ldg(pc++);
          uint32_t x1 = C.x(o.y), z1 = C.z(o.y), x2 = C.x(o.z), z2 = C.z(o.z);
          gate2_xz(o.x, x1, z1, x2, z2);
          C.x(o.y) = x1; C.z(o.y) = z1; C.x(o.z) = x2; C.z(o.z) = z2;
        }
        break;
      }
      case SEG_MZ: {
        for (uint32_t i = 0; i < cnt; i += 2) {
          const uint4 o = __ldg(pc++);
          uint32_t x0 = C.x(o.x), x1 = C.x(o.z);
          if (o.y != BIT_NONE) rec[(uint64_t)o.y * pitch] = x0;
          if (o.w != BIT_NONE) rec[(uint64_t)o.w * pitch] = x1;
        }
        break;
      }
      case SEG_MRZ: {
        for (uint32_t i = 0; i < cnt; i++) {
          const uint4 o = __ldg(pc++);  // (q, bit, reset index, 0)
          uint32_t x = C.x(o.x), z = C.z(o.x);
          uint32_t rb;
          if (PHILOX) {
            if ((o.z >> 2) != rblk) {
              rblk = o.z >> 2;
              philox4x32_10(rblk, clo, chi, TAG_RESET, k0, k1, rc);
            }
            rb = sel4(rc, o.z & 3);
          } else {
            rb = a.reset_planes ? __ldg(a.reset_planes + (uint64_t)o.z * a.reset_pitch + c) : 0u;
          }
          if (o.y != BIT_NONE) rec[(uint64_t)o.y * pitch] = x;
          C.x(o.x) = 0u;
          C.z(o.x) = z ^ rb;
        }
        break;
      }
      case SEG_FLUSH: {
        const uint64_t lim = (uint64_t)h.z * 32u;
        if (PHILOX) {
          while (ns.alive && ns.t < lim) {
            const uint32_t site = (uint32_t)(ns.t >> 5);
            const Site s = a.sites[site];
            const uint32_t code = site_code(s, ns.v);
            if (code) apply_event(C, s, code, 1u << (ns.t & 31));
            noise_step(ns, a, col, false);
          }
        } else {
          while (ep < ee) {
            const uint64_t d = __ldg(a.ev_data + ep);
            const uint64_t t = d >> 8;
            if (t >= lim) break;
            const Site s = a.sites[(uint32_t)(t >> 5)];
            apply_event(C, s, (uint32_t)(d & 0xFF), 1u << (t & 31));
            ep++;
          }
        }
        break;
      }
      default:
        return;
    }
  }
}

template <bool SMEM, bool PHILOX>
__global__ void __launch_bounds__(256) walker_kernel(const WalkArgs a) {
  extern __shared__ __align__(16) uint32_t sm[];
  const uint32_t NT = blockDim.x, tid = threadIdx.x;
  if (!SMEM) {
    for (uint32_t s = tid; s <= a.nslots; s += NT) sm[s] = s < a.nslots ? a.slot_qubit[s] : a.scratch_plane;
    __syncthreads();
  }
  const uint64_t ntiles = (a.ncols + NT - 1) / NT;
  for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const uint64_t c = tile * NT + tid;
    if (c >= a.ncols) break;
    const uint64_t col = a.col0 + c;
    const uint32_t k0 = (uint32_t)a.seed, k1 = (uint32_t)(a.seed >> 32);
    if (SMEM) {
      SmemCol C{sm + tid, NT};
      if (a.fresh) {
        for (uint32_t q = 0; q < a.nq1; q += 4) {
          uint32_t o[4];
          philox4x32_10(q >> 2, (uint32_t)col, (uint32_t)(col >> 32), TAG_INITZ, k0, k1, o);
#pragma unroll
          for (uint32_t j = 0; j < 4; j++) {
            const uint32_t qq = q + j;
            if (qq >= a.nq1) break;
            const uint32_t s = qq < a.qubit_slot_len ? __ldg(a.qubit_slot + qq) : BIT_NONE;
            if (s != BIT_NONE) {
              C.x(s) = 0u;
              C.z(s) = o[j];
            } else {
              a.planes[(uint64_t)(2 * qq) * a.pitch + c] = 0u;
              a.planes[(uint64_t)(2 * qq + 1) * a.pitch + c] = o[j];
            }
          }
        }
      } else {
        for (uint32_t s = 0; s < a.nslots; s++) {
          const uint32_t q = __ldg(a.slot_qubit + s);
          C.x(s) = a.planes[(uint64_t)(2 * q) * a.pitch + c];
          C.z(s) = a.planes[(uint64_t)(2 * q + 1) * a.pitch + c];
        }
      }
      walk_column<SmemCol, PHILOX>(a, C, c);
      for (uint32_t s = 0; s < a.nslots; s++) {
        const uint32_t q = __ldg(a.slot_qubit + s);
        a.planes[(uint64_t)(2 * q) * a.pitch + c] = C.x(s);
        a.planes[(uint64_t)(2 * q + 1) * a.pitch + c] = C.z(s);
      }
    } else {
      GlobCol C{a.planes + c, sm, a.pitch};
      if (a.fresh) {
        for (uint32_t q = 0; q < a.nq1; q += 4) {
          uint32_t o[4];
          philox4x32_10(q >> 2, (uint32_t)col, (uint32_t)(col >> 32), TAG_INITZ, k0, k1, o);
#pragma unroll
          for (uint32_t j = 0; j < 4; j++) {
            const uint32_t qq = q + j;
            if (qq >= a.nq1) break;
            a.planes[(uint64_t)(2 * qq) * a.pitch + c] = 0u;
            a.planes[(uint64_t)(2 * qq + 1) * a.pitch + c] = o[j];
          }
        }
      }
      walk_column<GlobCol, PHILOX>(a, C, c);
    }
  }
}

// initZ! on its own: x = 0, z = Philox (src/pauli_frames.jl:47-56).
__global__ void initz_kernel(uint32_t* planes, uint64_t pitch, uint64_t ncols, uint32_t nq1,
                             uint64_t seed, uint64_t col0) {
  const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncols) return;
  const uint64_t col = col0 + c;
  for (uint32_t q = 0; q < nq1; q += 4) {
    uint32_t o[4];
    philox4x32_10(q >> 2, (uint32_t)col, (uint32_t)(col >> 32), TAG_INITZ, (uint32_t)seed,
                  (uint32_t)(seed >> 32), o);
    for (uint32_t j = 0; j < 4 && q + j < nq1; j++) {
      planes[(uint64_t)(2 * (q + j)) * pitch + c] = 0u;
      planes[(uint64_t)(2 * (q + j) + 1) * pitch + c] = o[j];
    }
  }
}

// planes -> reference fastcolumn xzs (frames x W' uint64, frames contiguous).
__global__ void planes_to_xzs_kernel(const uint32_t* planes, uint64_t pitch, uint32_t nq1,
                                     uint64_t S, uint32_t Wp, uint64_t* xzs) {
  const uint64_t f = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t w = blockIdx.y;
  if (f >= S) return;
  const uint32_t half = Wp / 2, xz = w >= half ? 1 : 0, wq = w - xz * half;
  const uint64_t cw = f >> 5;
  const uint32_t lane = (uint32_t)(f & 31);
  uint64_t v = 0;
  for (uint32_t b = 0; b < 64; b++) {
    const uint32_t q = wq * 64 + b;
    if (q >= nq1) break;
    const uint32_t word = __ldg(planes + (uint64_t)(2 * q + xz) * pitch + cw);
    v |= (uint64_t)((word >> lane) & 1u) << b;
  }
  xzs[(uint64_t)w * S + f] = v;
}

// reference fastcolumn xzs -> planes.
__global__ void xzs_to_planes_kernel(const uint64_t* xzs, uint64_t S, uint32_t Wp, uint32_t nq1,
                                     uint64_t ncols, uint32_t* planes, uint64_t pitch) {
  const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t pl = blockIdx.y;  // plane index 2q + xz
  if (c >= ncols) return;
  const uint32_t q = pl >> 1, xz = pl & 1, half = Wp / 2;
  const uint64_t* src = xzs + (uint64_t)(xz * half + (q >> 6)) * S;
  uint32_t v = 0;
  for (uint32_t l = 0; l < 32; l++) {
    const uint64_t f = c * 32 + l;
    if (f >= S) break;
    v |= (uint32_t)((__ldg(src + f) >> (q & 63)) & 1ull) << l;
  }
  planes[(uint64_t)pl * pitch + c] = v;
}

// record planes -> Bool matrix (frames x nbits, column-major).
__global__ void record_to_bools_kernel(const uint32_t* rec, uint64_t pitch, uint64_t S,
                                       uint32_t nbits, uint8_t* out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;  // 4 frames per thread
  const uint32_t b = blockIdx.y;
  const uint64_t f = i * 4;
  if (f >= S) return;
  const uint32_t word = __ldg(rec + (uint64_t)b * pitch + (f >> 5));
  const uint32_t sh = (uint32_t)(f & 31);
  uint8_t* dst = out + (uint64_t)b * S + f;
  for (uint32_t k = 0; k < 4 && f + k < S; k++) dst[k] = (uint8_t)((word >> (sh + k)) & 1u);
}

}  // namespace qcb

using namespace qcb;

static int check_frame(const qcb_frame* f) {
  if (!f) return fail(QCB_EARG, "null frame");
  return QCB_OK;
}

extern "C" {

int qcb_frame_create(uint64_t frames, uint32_t qubits, uint32_t nbits, qcb_frame** out) {
  if (!out) return fail(QCB_EARG, "qcb_frame_create: null out");
  *out = nullptr;
  if (qubits >= (1u << 30)) return fail(QCB_EBOUNDS, "qcb_frame_create: too many qubits");
  qcb_frame* f = new qcb_frame();
  f->frames = frames;
  f->qubits = qubits;
  f->nq1 = qubits + 1;
  f->nbits = nbits;
  f->ncols = (frames + 31) / 32;
  f->pitch = std::max<uint64_t>(32, (f->ncols + 31) / 32 * 32);
  size_t pbytes = (size_t)2 * (f->nq1 + 1) * f->pitch * 4;
  size_t rbytes = (size_t)std::max<uint32_t>(nbits, 1) * f->pitch * 4;
  cudaError_t e = cudaMalloc(&f->planes, pbytes);
  if (e == cudaSuccess) e = cudaMalloc(&f->record, rbytes);
  if (e == cudaSuccess) e = cudaMemset(f->planes, 0, pbytes);
  if (e == cudaSuccess) e = cudaMemset(f->record, 0, rbytes);
  if (e != cudaSuccess) {
    cudaFree(f->planes); cudaFree(f->record);
    delete f;
    return cuda_fail(e, "qcb_frame_create");
  }
  *out = f;
  return QCB_OK;
}

int qcb_frame_destroy(qcb_frame* f) {
  if (!f) return QCB_OK;
  cudaFree(f->planes);
  cudaFree(f->record);
  delete f;
  return QCB_OK;
}

int qcb_frame_shape(const qcb_frame* f, uint64_t* frames, uint32_t* qubits, uint32_t* nbits) {
  if (int st = check_frame(f)) return st;
  if (frames) *frames = f->frames;
  if (qubits) *qubits = f->qubits;
  if (nbits) *nbits = f->nbits;
  return QCB_OK;
}

int qcb_frame_init_z(qcb_frame* f, uint64_t seed, uint64_t shot_offset, void* stream) {
  if (int st = check_frame(f)) return st;
  if (shot_offset % 32) return fail(QCB_EARG, "shot_offset must be a multiple of 32");
  if (!f->ncols) return QCB_OK;
  uint32_t nt = 256;
  initz_kernel<<<(unsigned)((f->ncols + nt - 1) / nt), nt, 0, S(stream)>>>(
      f->planes, f->pitch, f->ncols, f->nq1, seed, shot_offset / 32);
  QCB_LAUNCHED();
  return QCB_OK;
}

int qcb_frame_init_z_planes(qcb_frame* f, const uint32_t* z, void* stream) {
  if (int st = check_frame(f)) return st;
  if (!f->ncols) return QCB_OK;
  // x planes to zero, z planes from the caller (strided 2D copy)
  QCB_CUDA(cudaMemset2DAsync(f->planes, 2 * f->pitch * 4, 0, f->ncols * 4, f->nq1, S(stream)));
  QCB_CUDA(cudaMemcpy2DAsync(f->planes + f->pitch, 2 * f->pitch * 4, z, f->ncols * 4,
                             f->ncols * 4, f->nq1, cudaMemcpyHostToDevice, S(stream)));
  QCB_CUDA(cudaStreamSynchronize(S(stream)));
  return QCB_OK;
}

int qcb_frame_clear(qcb_frame* f, void* stream) {
  if (int st = check_frame(f)) return st;
  QCB_CUDA(cudaMemsetAsync(f->planes, 0, (size_t)2 * (f->nq1 + 1) * f->pitch * 4, S(stream)));
  QCB_CUDA(cudaMemsetAsync(f->record, 0, (size_t)std::max<uint32_t>(f->nbits, 1) * f->pitch * 4, S(stream)));
  return QCB_OK;
}

}  // extern "C"

namespace qcb {

// Launch configuration for the walker (shared-memory tile when the touched
// qubits of a tile of >= 64 columns fit, else HBM planes).
struct WalkConfig {
  bool smem;
  uint32_t nt;
  uint32_t grid;
  size_t smem_bytes;
};

static WalkConfig walk_config(const qcb_program* p, const qcb_frame* f, uint32_t nt_hint) {
  WalkConfig wc{};
  const size_t per_thread = (size_t)(p->nslots + 1) * 2 * 4;
  const size_t maxsm = (size_t)device_max_smem_optin();
  uint32_t nt = 0;
  for (uint32_t cand = 256; cand >= 64; cand -= 32)
    if (per_thread * cand <= maxsm) { nt = cand; break; }
  if (nt_hint && per_thread * nt_hint <= maxsm) nt = nt_hint;
  if (nt >= 64) {
    wc.smem = true;
    wc.nt = nt;
    wc.smem_bytes = per_thread * nt;
  } else {
    wc.smem = false;
    wc.nt = 128;
    wc.smem_bytes = (size_t)(p->nslots + 1) * 4;
  }
  uint64_t tiles = (f->ncols + wc.nt - 1) / wc.nt;
  wc.grid = (uint32_t)std::min<uint64_t>(tiles ? tiles : 1, 1u << 30);
  return wc;
}

static uint32_t g_nt_override = 0;

int launch_walker(qcb_frame* f, const qcb_program* p, WalkArgs& a, bool philox, bool fresh,
                  cudaStream_t st) {
  WalkConfig wc = walk_config(p, f, g_nt_override);
  a.fresh = fresh ? 1 : 0;
  if (!f->ncols) return QCB_OK;
  void (*kern)(const WalkArgs);
  if (wc.smem) kern = philox ? walker_kernel<true, true> : walker_kernel<true, false>;
  else kern = philox ? walker_kernel<false, true> : walker_kernel<false, false>;
  if (wc.smem_bytes > 48 * 1024)
    QCB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wc.smem_bytes));
  kern<<<wc.grid, wc.nt, wc.smem_bytes, st>>>(a);
  QCB_LAUNCHED();
  return QCB_OK;
}

static void fill_common(WalkArgs& a, qcb_frame* f, const qcb_program* p) {
  std::memset(&a, 0, sizeof(a));
  a.prog = (const uint4*)p->d_stream_slot;
  a.planes = f->planes;
  a.rec = f->record;
  a.pitch = f->pitch;
  a.ncols = f->ncols;
  a.slot_qubit = p->d_slot_qubit;
  a.nslots = p->nslots;
  a.scratch_plane = f->nq1;
  a.nq1 = f->nq1;
  a.qubit_slot = p->d_qubit_slot;
  a.qubit_slot_len = p->qubit_slot_len;
  a.nsites = p->info.n_noise_sites;
  a.sites = p->d_sites_slot;
  a.pmax = p->pmax;
  a.inv_log1m = p->inv_log1m;
}

static int check_run(const qcb_frame* f, const qcb_program* p, const qcb_noise_source* n) {
  if (!f || !p || !n) return fail(QCB_EARG, "null argument");
  if (p->nq > f->nq1)
    return fail(QCB_EBOUNDS, "program uses qubit " + std::to_string(p->nq) + " but the frame has " +
                                 std::to_string(f->nq1) + " (qubits + hidden ancilla)");
  if (p->info.nbits > f->nbits)
    return fail(QCB_EBOUNDS, "program records bit " + std::to_string(p->info.nbits) +
                                 " but the frame has " + std::to_string(f->nbits));
  if (n->shot_offset % 32) return fail(QCB_EARG, "shot_offset must be a multiple of 32");
  if (n->mode != QCB_NOISE_PHILOX && n->mode != QCB_NOISE_MASK) return fail(QCB_EARG, "bad noise mode");
  return QCB_OK;
}

int run_program(qcb_frame* f, const qcb_program* p, const qcb_noise_source* n, bool fresh,
                cudaStream_t st) {
  if (int s = check_run(f, p, n)) return s;
  WalkArgs a;
  fill_common(a, f, p);
  a.seed = n->seed;
  a.col0 = n->shot_offset / 32;
  if (n->mode == QCB_NOISE_PHILOX) return launch_walker(f, p, a, true, fresh, st);

  // Mask mode: bucket the caller's events per column, sorted by trial.
  const uint64_t ncols = f->ncols;
  std::vector<uint64_t> off(ncols + 1, 0);
  std::vector<std::pair<uint64_t, uint64_t>> evs;  // (column, data)
  evs.reserve(n->n_events);
  for (uint64_t i = 0; i < n->n_events; i++) {
    const qcb_event& e = n->events[i];
    if (e.op_index >= p->site_of_op.size() || p->site_of_op[e.op_index] < 0)
      return fail(QCB_EARG, "event " + std::to_string(i) + ": op_index is not a noise op");
    if (e.shot >= f->frames) return fail(QCB_EBOUNDS, "event " + std::to_string(i) + ": shot out of range");
    const uint64_t site = (uint64_t)p->site_of_op[e.op_index];
    const uint32_t ar = p->site_arity[site];
    const uint32_t maxcode = ar == 2 ? 15u : 3u;
    if (e.pauli > maxcode) return fail(QCB_EARG, "event " + std::to_string(i) + ": bad Pauli code");
    if (e.pauli == 0) continue;
    const uint64_t t = site * 32 + (e.shot & 31);
    evs.push_back({e.shot >> 5, (t << 8) | e.pauli});
  }
  std::sort(evs.begin(), evs.end());
  for (auto& e : evs) off[e.first + 1]++;
  for (uint64_t c = 0; c < ncols; c++) off[c + 1] += off[c];
  std::vector<uint64_t> data(evs.size());
  for (size_t i = 0; i < evs.size(); i++) data[i] = evs[i].second;
  uint64_t *d_off = nullptr, *d_data = nullptr;
  uint32_t* d_reset = nullptr;
  QCB_CUDA(cudaMallocAsync(&d_off, off.size() * 8, st));
  QCB_CUDA(cudaMallocAsync(&d_data, std::max<size_t>(data.size(), 1) * 8, st));
  QCB_CUDA(cudaMemcpyAsync(d_off, off.data(), off.size() * 8, cudaMemcpyHostToDevice, st));
  if (!data.empty())
    QCB_CUDA(cudaMemcpyAsync(d_data, data.data(), data.size() * 8, cudaMemcpyHostToDevice, st));
  if (n->reset_planes && p->info.n_resets) {
    size_t bytes = (size_t)p->info.n_resets * ncols * 4;
    QCB_CUDA(cudaMallocAsync(&d_reset, bytes, st));
    QCB_CUDA(cudaMemcpyAsync(d_reset, n->reset_planes, bytes, cudaMemcpyHostToDevice, st));
  }
  a.ev_off = d_off;
  a.ev_data = d_data;
  a.reset_planes = d_reset;
  a.reset_pitch = ncols;
  int s = launch_walker(f, p, a, false, fresh, st);
  // host vectors must outlive the async copies
  cudaError_t e = cudaStreamSynchronize(st);
  cudaFreeAsync(d_off, st);
  cudaFreeAsync(d_data, st);
  if (d_reset) cudaFreeAsync(d_reset, st);
  if (e != cudaSuccess) return cuda_fail(e, "pftrajectories (mask mode)");
  return s;
}

}  // namespace qcb

extern "C" {

int qcb_pftrajectories(qcb_frame* f, const qcb_program* p, const qcb_noise_source* n, void* stream) {
  return run_program(f, p, n, false, S(stream));
}

int qcb_frame_apply_ops(qcb_frame* f, const qcb_op* ops, size_t n_ops, const qcb_noise_source* n,
                        void* stream) {
  qcb_program* p = nullptr;
  if (int st = qcb_program_compile(ops, n_ops, &p)) return st;
  int st = run_program(f, p, n, false, S(stream));
  cudaStreamSynchronize(S(stream));
  qcb_program_destroy(p);
  return st;
}

int qcb_frame_download_xzs(const qcb_frame* f, uint64_t* xzs, void* stream) {
  if (int st = check_frame(f)) return st;
  const uint32_t Wp = 2 * ((f->nq1 + 63) / 64);
  const size_t bytes = (size_t)Wp * f->frames * 8;
  if (!bytes) return QCB_OK;
  uint64_t* d = nullptr;
  QCB_CUDA(cudaMallocAsync(&d, bytes, S(stream)));
  dim3 grid((unsigned)((f->frames + 255) / 256), Wp);
  planes_to_xzs_kernel<<<grid, 256, 0, S(stream)>>>(f->planes, f->pitch, f->nq1, f->frames, Wp, d);
  QCB_LAUNCHED();
  QCB_CUDA(cudaMemcpyAsync(xzs, d, bytes, cudaMemcpyDeviceToHost, S(stream)));
  QCB_CUDA(cudaFreeAsync(d, S(stream)));
  QCB_CUDA(cudaStreamSynchronize(S(stream)));
  return QCB_OK;
}

int qcb_frame_upload_xzs(qcb_frame* f, const uint64_t* xzs, void* stream) {
  if (int st = check_frame(f)) return st;
  const uint32_t Wp = 2 * ((f->nq1 + 63) / 64);
  const size_t bytes = (size_t)Wp * f->frames * 8;
  if (!bytes) return QCB_OK;
  uint64_t* d = nullptr;
  QCB_CUDA(cudaMallocAsync(&d, bytes, S(stream)));
  QCB_CUDA(cudaMemcpyAsync(d, xzs, bytes, cudaMemcpyHostToDevice, S(stream)));
  dim3 grid((unsigned)((f->ncols + 255) / 256), 2 * f->nq1);
  xzs_to_planes_kernel<<<grid, 256, 0, S(stream)>>>(d, f->frames, Wp, f->nq1, f->ncols, f->planes, f->pitch);
  QCB_LAUNCHED();
  QCB_CUDA(cudaFreeAsync(d, S(stream)));
  QCB_CUDA(cudaStreamSynchronize(S(stream)));
  return QCB_OK;
}

int qcb_frame_download_measurements(const qcb_frame* f, uint8_t* bools, void* stream) {
  if (int st = check_frame(f)) return st;
  const size_t bytes = (size_t)f->frames * f->nbits;
  if (!bytes) return QCB_OK;
  uint8_t* d = nullptr;
  QCB_CUDA(cudaMallocAsync(&d, bytes, S(stream)));
  dim3 grid((unsigned)(((f->frames + 3) / 4 + 255) / 256), f->nbits);
  record_to_bools_kernel<<<grid, 256, 0, S(stream)>>>(f->record, f->pitch, f->frames, f->nbits, d);
  QCB_LAUNCHED();
  QCB_CUDA(cudaMemcpyAsync(bools, d, bytes, cudaMemcpyDeviceToHost, S(stream)));
  QCB_CUDA(cudaFreeAsync(d, S(stream)));
  QCB_CUDA(cudaStreamSynchronize(S(stream)));
  return QCB_OK;
}

int qcb_frame_download_record_planes(const qcb_frame* f, uint32_t* planes, void* stream) {
  if (int st = check_frame(f)) return st;
  if (!f->nbits || !f->ncols) return QCB_OK;
  QCB_CUDA(cudaMemcpy2DAsync(planes, f->ncols * 4, f->record, f->pitch * 4, f->ncols * 4, f->nbits,
                             cudaMemcpyDeviceToHost, S(stream)));
  QCB_CUDA(cudaStreamSynchronize(S(stream)));
  return QCB_OK;
}

int qcb_frame_download_planes(const qcb_frame* f, uint32_t* xp, uint32_t* zp, void* stream) {
  if (int st = check_frame(f)) return st;
  if (!f->ncols) return QCB_OK;
  if (xp)
    QCB_CUDA(cudaMemcpy2DAsync(xp, f->ncols * 4, f->planes, 2 * f->pitch * 4, f->ncols * 4, f->nq1,
                               cudaMemcpyDeviceToHost, S(stream)));
  if (zp)
    QCB_CUDA(cudaMemcpy2DAsync(zp, f->ncols * 4, f->planes + f->pitch, 2 * f->pitch * 4, f->ncols * 4,
                               f->nq1, cudaMemcpyDeviceToHost, S(stream)));
  QCB_CUDA(cudaStreamSynchronize(S(stream)));
  return QCB_OK;
}

// One-call pftrajectories(circuit; trajectories): program and frame are
// cached between calls (keyed by the op list and the frame shape).
int qcb_pftrajectories_host(const qcb_op* ops, size_t n_ops, uint64_t frames, uint64_t seed,
                            uint64_t shot_offset, uint32_t* record_planes, void* stream) {
  static std::mutex mu;
  static qcb_program* cprog = nullptr;
  static std::vector<qcb_op> cops;
  static qcb_frame* cframe = nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!cprog || cops.size() != n_ops || std::memcmp(cops.data(), ops, n_ops * sizeof(qcb_op)) != 0) {
    if (cprog) { qcb_program_destroy(cprog); cprog = nullptr; }
    if (int st = qcb_program_compile(ops, n_ops, &cprog)) return st;
    cops.assign(ops, ops + n_ops);
  }
  // _create_pauliframe: qmax / bmax with init = 1 (src/pauli_frames.jl:197-201)
  const uint32_t qmax = std::max<uint32_t>(cprog->info.nqubits, 1);
  const uint32_t bmax = std::max<uint32_t>(cprog->info.nbits, 1);
  if (!cframe || cframe->frames != frames || cframe->qubits != qmax || cframe->nbits != bmax) {
    if (cframe) { qcb_frame_destroy(cframe); cframe = nullptr; }
    if (int st = qcb_frame_create(frames, qmax, bmax, &cframe)) return st;
  }
  qcb_noise_source n{};
  n.mode = QCB_NOISE_PHILOX;
  n.seed = seed;
  n.shot_offset = shot_offset;
  if (int st = run_program(cframe, cprog, &n, true, S(stream))) return st;
  if (record_planes) return qcb_frame_download_record_planes(cframe, record_planes, stream);
  return QCB_OK;
}

}  // extern "C"

extern "C" int qcb_pftrajectories_fresh(qcb_frame* f, const qcb_program* p, uint64_t seed,
                                        uint64_t shot_offset, void* stream) {
  qcb_noise_source n{};
  n.mode = QCB_NOISE_PHILOX;
  n.seed = seed;
  n.shot_offset = shot_offset;
  return run_program(f, p, &n, true, S(stream));
}

// Internal hooks for the batched runner and the tuner.
namespace qcb {
void set_walker_nt(uint32_t nt) { g_nt_override = nt; }
int run_program_fresh(qcb_frame* f, const qcb_program* p, uint64_t seed, uint64_t shot_offset,
                      cudaStream_t st) {
  qcb_noise_source n{};
  n.mode = QCB_NOISE_PHILOX;
  n.seed = seed;
  n.shot_offset = shot_offset;
  return run_program(f, p, &n, true, st);
}
}  // namespace qcb
