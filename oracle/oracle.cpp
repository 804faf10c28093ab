// oracle.cpp -- CPU restatement of QuantumClifford.jl v0.11.7's bit-packed
// tableau and Pauli-frame hot path, in the reference's own data layout.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, the smoke()
// entry and the CPU-baseline leg of bench.py load it to compare against or to
// time beside the CUDA library.  Nothing in the product links or calls it.
//
// Parity pins: tests/test_oracle_golden.py checks every function here against
// the known answers written in the reference's doctests and tests (cited
// there).  The Pauli-frame RNG streams of the reference (Julia's task-local
// Xoshiro256++) cannot be reproduced, so frame parity uses "mask mode": both
// this oracle and the device consume the same seeded event file.
//
// Layouts (as in the reference):
//  - Tableau (src/QuantumClifford.jl:145-151): row r is W = 2*ceil(n/64)
//    uint64 words at xzs + r*W, X words then Z words; phases uint8 mod 4.
//  - PauliFrame (src/pauli_frames.jl:30-37, fastcolumn): the frame tableau's
//    xzs is the Adjoint of an (S x W') matrix, so element (frame f, word w)
//    lives at xzs[w*S + f]; W' = 2*ceil((n+1)/64).
//  - Record: Bool matrix S x nbits, column-major: meas[(b-1)*S + f].
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>
#include <algorithm>

#include "../include/qcb200.h"

typedef uint64_t u64;
typedef uint32_t u32;
typedef uint8_t u8;

static inline int popc64(u64 x) { return __builtin_popcountll(x); }

// ---------------------------------------------------------------- RNG
// Xoshiro256++ (Blackman & Vigna), the generator behind Julia's default
// task-local RNG; used for the reference-structured CPU baseline and for the
// statistical comparisons.  Seeded with SplitMix64.
struct Xoshiro {
  u64 s[4];
  static inline u64 rotl(u64 x, int k) { return (x << k) | (x >> (64 - k)); }
  explicit Xoshiro(u64 seed) {
    for (int i = 0; i < 4; i++) {
      seed += 0x9E3779B97F4A7C15ull;
      u64 z = seed;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      s[i] = z ^ (z >> 31);
    }
  }
  inline u64 next() {
    u64 r = rotl(s[0] + s[3], 23) + s[0];
    u64 t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t; s[3] = rotl(s[3], 45);
    return r;
  }
  inline double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }
};

// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11): 10 rounds of the 4x32 Philox S-box with the
// published multipliers and Weyl key increments.
extern "C" void oracle_philox4x32_10(const u32 ctr_in[4], const u32 key_in[2], u32 out[4]) {
  u32 c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  u32 k0 = key_in[0], k1 = key_in[1];
  for (int r = 0; r < 10; r++) {
    u64 p0 = (u64)0xD2511F53u * c0;
    u64 p1 = (u64)0xCD9E8D57u * c2;
    u32 n0 = (u32)(p1 >> 32) ^ c1 ^ k0;
    u32 n1 = (u32)p1;
    u32 n2 = (u32)(p0 >> 32) ^ c3 ^ k1;
    u32 n3 = (u32)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// ---------------------------------------------------------------- gate tables
// Symbolic gate truth tables, src/symbolic_cliffords.jl:105-118 (1q) and
// :358-395 (2q).  Bit-sliced: every argument is a word of independent lanes.
// Returns the phase flag word (lanes whose phase gains +2).
static inline u64 gate1(u32 op, u64& x, u64& z) {
  u64 X = x, Z = z, ph = 0;
  if ((op & 0xFF) == QCB_OP_SQO) {
    // SingleQubitOperator (src/symbolic_cliffords.jl:178-206); flags in op >> 8:
    // xx, xz, zx, zz, px, pz
    u32 f = op >> 8;
    bool xx = f & 1, xz = f & 2, zx = f & 4, zz = f & 8, px = f & 16, pz = f & 32;
    bool anticom = (!zz && xz && !xx && zx) || (zz && !xz && xx && zx) || (zz && xz && xx && !zx);
    x = (xx ? X : 0) ^ (zx ? Z : 0);
    z = (xz ? X : 0) ^ (zz ? Z : 0);
    return (px ? X : 0) ^ (pz ? Z : 0) ^ (anticom ? (X & Z) : 0);
  }
  switch (op) {
    case QCB_OP_I: break;
    case QCB_OP_H: x = Z; z = X; ph = X & Z; break;
    case QCB_OP_HXY: x = X; z = X ^ Z; ph = ~X & Z; break;
    case QCB_OP_HYZ: x = X ^ Z; z = Z; ph = X & ~Z; break;
    case QCB_OP_S: x = X; z = X ^ Z; ph = X & Z; break;
    case QCB_OP_SDAG: x = X; z = X ^ Z; ph = X & ~Z; break;
    case QCB_OP_X: ph = Z; break;
    case QCB_OP_Y: ph = X ^ Z; break;
    case QCB_OP_Z: ph = X; break;
    case QCB_OP_SQRTX: x = X ^ Z; z = Z; ph = ~X & Z; break;
    case QCB_OP_INVSQRTX: x = X ^ Z; z = Z; ph = X & Z; break;
    case QCB_OP_SQRTY: x = Z; z = X; ph = X & ~Z; break;
    case QCB_OP_INVSQRTY: x = Z; z = X; ph = Z & ~X; break;
    case QCB_OP_CXYZ: x = X ^ Z; z = X; break;
    case QCB_OP_CZYX: x = Z; z = X ^ Z; break;
    default: break;
  }
  return ph;
}

static inline u64 gate2(u32 op, u64& x1, u64& z1, u64& x2, u64& z2) {
  u64 a = x1, b = z1, c = x2, d = z2, ph = 0;  // a=x1 b=z1 c=x2 d=z2
  switch (op) {
    case QCB_OP_SWAP: x1 = c; z1 = d; x2 = a; z2 = b; break;
    case QCB_OP_CNOT:
      x1 = a; z1 = b ^ d; x2 = c ^ a; z2 = d;
      ph = (a & b & c & d) | (a & d & ~(b | c)); break;
    case QCB_OP_CPHASE:
      x1 = a; z1 = b ^ c; x2 = c; z2 = d ^ a;
      ph = (a & b & c & ~d) | (a & ~b & c & d); break;
    case QCB_OP_ZCX:
      x1 = a; z1 = b ^ d; x2 = c ^ a; z2 = d;
      ph = (a & d) & ~(b ^ c); break;
    case QCB_OP_ZCY:
      x1 = a; z1 = c ^ b ^ d; x2 = c ^ a; z2 = d ^ a;
      ph = a & (c ^ b) & (c ^ d); break;
    case QCB_OP_ZCZ:
      x1 = a; z1 = b ^ c; x2 = c; z2 = d ^ a;
      ph = (b ^ d) & (a & c); break;
    case QCB_OP_XCX:
      x1 = d ^ a; z1 = b; x2 = c ^ b; z2 = d;
      ph = (b & d) & (a ^ c); break;
    case QCB_OP_XCY:
      x1 = a ^ c ^ d; z1 = b; x2 = b ^ c; z2 = d ^ b;
      ph = b & (c ^ d) & ~(c ^ a); break;
    case QCB_OP_XCZ:
      x1 = a ^ c; z1 = b; x2 = c; z2 = d ^ b;
      ph = (c & b) & ~(a ^ d); break;
    case QCB_OP_YCX:
      x1 = a ^ d; z1 = d ^ b; x2 = a ^ b ^ c; z2 = d;
      ph = d & (a ^ b) & ~(c ^ a); break;
    case QCB_OP_YCY:
      x1 = a ^ d ^ c; z1 = b ^ c ^ d; x2 = a ^ c ^ b; z2 = a ^ b ^ d;
      ph = (a & ~b & ~c & d) | (~a & b & c & ~d); break;
    case QCB_OP_YCZ:
      x1 = a ^ c; z1 = c ^ b; x2 = c; z2 = d ^ a ^ b;
      ph = c & (a ^ b) & (d ^ a); break;
    // src/symbolic_cliffords.jl:361-395
    case QCB_OP_SWAPCX:
      x1 = c; z1 = d ^ b; x2 = c ^ a; z2 = b;
      ph = (a & b & c & d) | (~a & b & c & ~d); break;
    case QCB_OP_INVSWAPCX:
      x1 = c ^ a; z1 = d; x2 = a; z2 = d ^ b;
      ph = (a & b & c & d) | (a & ~b & ~c & d); break;
    case QCB_OP_ISWAP:
      x1 = c; z1 = a ^ d ^ c; x2 = a; z2 = a ^ c ^ b;
      ph = (a & b & ~c) | (~a & c & d); break;
    case QCB_OP_INVISWAP:
      x1 = c; z1 = a ^ d ^ c; x2 = a; z2 = a ^ c ^ b;
      ph = (a & ~b & ~c) | (~a & c & ~d); break;
    case QCB_OP_CZSWAP:
      x1 = c; z1 = d ^ a; x2 = a; z2 = c ^ b;
      ph = (a & ~b & c & d) | (a & b & c & ~d); break;
    case QCB_OP_CXSWAP:
      x1 = c ^ a; z1 = d; x2 = a; z2 = d ^ b;
      ph = (a & ~b & ~c & d) | (a & b & c & d); break;
    case QCB_OP_ZCRY:
      x1 = a; z1 = a ^ b ^ c ^ d; x2 = a ^ c; z2 = a ^ d;
      ph = (a & ~b & c) | (a & ~b & ~d) | (a & c & ~d); break;
    case QCB_OP_INVZCRY:
      x1 = a; z1 = a ^ b ^ c ^ d; x2 = a ^ c; z2 = a ^ d;
      ph = (a & b & ~c) | (a & b & d) | (a & ~c & d); break;
    case QCB_OP_SQRTZZ:
      x1 = a; z1 = a ^ c ^ b; x2 = c; z2 = a ^ d ^ c;
      ph = (a & b & ~c) | (~a & c & d); break;
    case QCB_OP_INVSQRTZZ:
      x1 = a; z1 = a ^ c ^ b; x2 = c; z2 = a ^ d ^ c;
      ph = (a & ~b & ~c) | (~a & c & ~d); break;
    case QCB_OP_SQRTXX:
      x1 = b ^ d ^ a; z1 = b; x2 = b ^ c ^ d; z2 = d;
      ph = (~a & b & ~d) | (~b & ~c & d); break;
    case QCB_OP_INVSQRTXX:
      x1 = b ^ d ^ a; z1 = b; x2 = b ^ c ^ d; z2 = d;
      ph = (a & b & ~d) | (~b & c & d); break;
    case QCB_OP_SQRTYY:
      x1 = b ^ c ^ d; z1 = a ^ d ^ c; x2 = a ^ b ^ d; z2 = a ^ c ^ b;
      ph = (~a & ~b & c & ~d) | (a & ~b & ~c & ~d) | (a & ~b & c & d) | (a & b & c & ~d); break;
    case QCB_OP_INVSQRTYY:
      x1 = b ^ c ^ d; z1 = a ^ d ^ c; x2 = a ^ b ^ d; z2 = a ^ c ^ b;
      ph = (a & b & ~c & d) | (~a & b & c & d) | (~a & b & ~c & ~d) | (~a & ~b & ~c & d); break;
    default: break;
  }
  return ph;
}

static inline bool is1q(u32 op) { return op >= QCB_OP_I && op <= QCB_OP_SQO; }
// gate code of a 1-qubit op: SingleQubitOperator carries its flags (q2) along
static inline u32 code1(const qcb_op& op) {
  return op.opcode == QCB_OP_SQO ? op.opcode | ((op.q2 & 63u) << 8) : op.opcode;
}
static inline bool is2q(u32 op) { return op >= QCB_OP_CNOT && op <= QCB_OP_LAST2Q; }

// ---------------------------------------------------------------- Pauli rows
// mul_left!(r, l) on raw words (src/mul_leftright.jl:11-31 / 75-126): r ^= l
// with the Stim phase counters; returns the extra phase (0..3).
static inline u8 row_mul_left(u64* r, const u64* l, size_t W, bool phases) {
  size_t len = W / 2;
  if (!phases) {
    for (size_t i = 0; i < W; i++) r[i] ^= l[i];
    return 0;
  }
  u64 cnt1 = 0, cnt2 = 0;
  for (size_t i = 0; i < len; i++) {
    u64 x1 = l[i], x2 = r[i], z1 = l[i + len], z2 = r[i + len];
    u64 newx1 = x1 ^ x2, newz1 = z1 ^ z2;
    r[i] = newx1; r[i + len] = newz1;
    u64 x1z2 = x1 & z2;
    u64 anti = (x2 & z1) ^ x1z2;
    cnt2 ^= (cnt1 ^ newx1 ^ newz1 ^ x1z2) & anti;
    cnt1 ^= anti;
  }
  int c1 = popc64(cnt1), c2 = popc64(cnt2);
  return (u8)((c1 ^ (c2 << 1)) & 3);
}

// prodphase (src/QuantumClifford.jl:723-733).
static inline u8 row_prodphase(const u64* l, const u64* r, size_t W) {
  long res = 0;
  size_t len = W / 2;
  for (size_t i = 0; i < len; i++) {
    u64 x1 = l[i], x2 = r[i], z1 = l[i + len], z2 = r[i + len];
    res += popc64((~z2 & x2 & ~x1 & z1) | (z2 & ~x2 & x1 & z1) | (z2 & x2 & x1 & ~z1));
    res -= popc64((z2 & x2 & ~x1 & z1) | (~z2 & x2 & x1 & z1) | (z2 & ~x2 & x1 & ~z1));
  }
  return (u8)((u64)res & 3);
}

// comm (src/QuantumClifford.jl:791-798).
static inline u8 row_comm(const u64* l, const u64* r, size_t W) {
  u64 res = 0;
  size_t len = W / 2;
  for (size_t i = 0; i < len; i++) res ^= (l[i + len] & r[i]) ^ (l[i] & r[i + len]);
  return (u8)(popc64(res) & 1);
}

struct Tab {
  u64* xzs; u8* ph; size_t W; u32 n;
  u64* row(size_t r) const { return xzs + r * W; }
  bool xbit(size_t r, u32 q) const { return (row(r)[q >> 6] >> (q & 63)) & 1; }
  bool zbit(size_t r, u32 q) const { return (row(r)[W / 2 + (q >> 6)] >> (q & 63)) & 1; }
};

// mul_left!(s::Tableau, m, i) (src/mul_leftright.jl:177-181): row m <- row i * row m.
static inline void tab_mul_left(Tab& t, size_t m, size_t i, bool phases) {
  u8 e = row_mul_left(t.row(m), t.row(i), t.W, phases);
  if (phases) t.ph[m] = (u8)((e + t.ph[m] + t.ph[i]) & 3);
}

// rowswap! (src/QuantumClifford.jl:899-905).
static inline void tab_rowswap(Tab& t, size_t i, size_t j, bool phases) {
  if (i == j) return;
  if (phases) std::swap(t.ph[i], t.ph[j]);
  for (size_t k = 0; k < t.W; k++) std::swap(t.row(i)[k], t.row(j)[k]);
}

static inline void tab_setrow(Tab& t, size_t m, const u64* xz, u8 phase) {
  std::memcpy(t.row(m), xz, t.W * 8);
  t.ph[m] = phase;
}

extern "C" {

u8 oracle_mul_left_words(u64* r, const u64* l, size_t W, int phases) {
  return row_mul_left(r, l, W, phases != 0);
}

// mul_left!(r::PauliOperator, l::PauliOperator) (src/mul_leftright.jl:137-142).
void oracle_mul_left_pauli(u64* r, u8* r_phase, const u64* l, u8 l_phase, size_t W, int phases) {
  u8 s = row_mul_left(r, l, W, phases != 0);
  if (phases) *r_phase = (u8)((s + *r_phase + l_phase) & 3);
}

u8 oracle_prodphase(const u64* l, const u64* r, size_t W) { return row_prodphase(l, r, W); }
u8 oracle_comm(const u64* l, const u64* r, size_t W) { return row_comm(l, r, W); }

// mul_right!(l, r) on words (src/mul_leftright.jl:128-131): l ^= r through
// mul_ordered!(l, r) and the phase ((rcnt1 ^ (rcnt2 << 1)) + 2 rcnt1) & 3.
static inline u8 row_mul_right(u64* l, const u64* r, size_t W, bool phases) {
  size_t len = W / 2;
  if (!phases) {
    for (size_t i = 0; i < W; i++) l[i] ^= r[i];
    return 0;
  }
  u64 cnt1 = 0, cnt2 = 0;
  for (size_t i = 0; i < len; i++) {
    u64 x1 = r[i], x2 = l[i], z1 = r[i + len], z2 = l[i + len];
    u64 newx1 = x1 ^ x2, newz1 = z1 ^ z2;
    l[i] = newx1; l[i + len] = newz1;
    u64 x1z2 = x1 & z2;
    u64 anti = (x2 & z1) ^ x1z2;
    cnt2 ^= (cnt1 ^ newx1 ^ newz1 ^ x1z2) & anti;
    cnt1 ^= anti;
  }
  int c1 = popc64(cnt1), c2 = popc64(cnt2);
  return (u8)(((c1 ^ (c2 << 1)) + c1 * 2) & 3);
}

// The mul_left!/mul_right! family on rows, one reference call per target
// row, in order (src/mul_leftright.jl:137-245): s[a] <- t[b] * s[a]
// (right = 0) or s[a] * t[b] (right = 1), a = s_row + k, b = t_row + k*t_step
// (1-based), phase (extra + s.phases[a] + P) & 3 with P = t.phases[b]
// (phase_src 0) or s.phases[b] (phase_src 1, :171-175, 183-187).
void oracle_mul_rows(u64* s_xz, u8* s_ph, const u64* t_xz, const u8* t_ph, size_t W, size_t s_row,
                     size_t count, size_t t_row, size_t t_step, int right, int phase_src, int phases) {
  std::vector<u64> src(W);
  for (size_t k = 0; k < count; k++) {
    size_t a = s_row - 1 + k, b = t_row - 1 + k * t_step;
    std::copy(t_xz + b * W, t_xz + (b + 1) * W, src.begin());  // as the reference's view reads it
    u8 add = phase_src ? s_ph[b] : t_ph[b];
    u8 e = right ? row_mul_right(s_xz + a * W, src.data(), W, phases != 0)
                 : row_mul_left(s_xz + a * W, src.data(), W, phases != 0);
    if (phases) s_ph[a] = (u8)((e + s_ph[a] + add) & 3);
  }
}

void oracle_mul_left_row(u64* xzs, u8* ph, size_t W, size_t m, size_t i, int phases) {
  Tab t{xzs, ph, W, 0};
  tab_mul_left(t, m - 1, i - 1, phases != 0);
}

// mul_left!(s::Tableau, p::PauliOperator) (src/mul_leftright.jl:221-227).
void oracle_mul_left_tableau_pauli(u64* xzs, u8* ph, size_t rows, size_t W, const u64* p,
                                   u8 p_phase, int phases) {
  for (size_t m = 0; m < rows; m++) {
    u8 e = row_mul_left(xzs + m * W, p, W, phases != 0);
    if (phases) ph[m] = (u8)((e + ph[m] + p_phase) & 3);
  }
}

// _canonicalize! (src/canonicalization.jl:95-133) on rows [0, rows).
void oracle_canonicalize(u64* xzs, u8* ph, size_t rows, u32 n, int phases, int* rx_out,
                         int* rz_out) {
  size_t W = 2 * ((n + 63) / 64);
  Tab t{xzs, ph, W, n};
  bool P = phases != 0;
  size_t i = 0;  // 0-based next pivot row
  for (int stage = 0; stage < 2; stage++) {
    for (u32 j = 0; j < n; j++) {
      size_t k = rows;
      for (size_t ii = i; ii < rows; ii++) {
        bool b = stage == 0 ? t.xbit(ii, j) : t.zbit(ii, j);
        if (b) { k = ii; break; }
      }
      if (k == rows) continue;
      tab_rowswap(t, k, i, P);
      for (size_t m = 0; m < rows; m++) {
        bool b = stage == 0 ? t.xbit(m, j) : t.zbit(m, j);
        if (b && m != i) tab_mul_left(t, m, i, P);
      }
      i++;
    }
    if (stage == 0 && rx_out) *rx_out = (int)i;  // rx - 1 in 1-based terms
  }
  if (rz_out) *rz_out = (int)i;
}

// _generate! (src/project_trace_reset.jl:41-81).  Returns 1 on success (the
// Pauli was generated; `p` now holds the identity up to a phase), 0 for
// `nothing`.  `used` receives 1-based row indices.
int oracle_generate(u64* p, u8* p_phase, const u64* xzs, const u8* ph, size_t rows, u32 n,
                    int phases, int* used, size_t* n_used) {
  size_t W = 2 * ((n + 63) / 64), len = W / 2;
  size_t u = 0;  // rows 1..u already consumed (1-based `used`)
  size_t nu = 0;
  for (int stage = 0; stage < 2; stage++) {
    while (true) {
      // first set bit of the X (stage 0) or Z (stage 1) half
      long bit = -1;
      for (size_t w = 0; w < len; w++) {
        u64 v = p[stage * len + w];
        if (v) { bit = (long)(w * 64 + __builtin_ctzll(v)); break; }
      }
      if (bit < 0) break;
      size_t ibig = (size_t)bit >> 6;
      u64 m = 1ull << (bit & 63);
      size_t cand = rows;
      for (size_t r = u; r < rows; r++) {
        if (xzs[r * W + stage * len + ibig] & m) { cand = r; break; }
      }
      if (cand == rows) { if (n_used) *n_used = nu; return 0; }
      u = cand + 1;
      u8 e = row_mul_left(p, xzs + cand * W, W, phases != 0);
      if (phases) *p_phase = (u8)((e + *p_phase + ph[cand]) & 3);
      if (used) used[nu] = (int)u;
      nu++;
    }
  }
  if (n_used) *n_used = nu;
  for (size_t w = 0; w < W; w++) if (p[w]) return 0;
  return 1;
}

// anticomm_update_rows (src/project_trace_reset.jl:319-335); 0-based rows,
// r = rank, nn = length (rows of each half), a = 1-based anticommuting index.
static void anticomm_update_rows(Tab& t, const u64* p, size_t r, size_t nn, size_t a, bool P) {
  size_t piv = nn + a - 1;
  for (size_t i = r; i < nn; i++)
    if (row_comm(p, t.row(i), t.W)) tab_mul_left(t, i, piv, P);
  for (size_t i = nn + a; i < 2 * nn; i++)
    if (row_comm(p, t.row(i), t.W)) tab_mul_left(t, i, piv, P);
  for (size_t i = 0; i < r; i++)
    if (i != a - 1 && row_comm(p, t.row(i), t.W)) tab_mul_left(t, i, piv, false);
}

// project! for the four tableau kinds (src/project_trace_reset.jl:276-439).
// rows: rows of the tableau buffer.  *rank_io is used for the mixed kinds.
// anticom: 1-based index or 0; result: 0..3 or -1 for `nothing`.
// Returns QCB_OK or QCB_EBADSTRUCT.
int oracle_project(int kind, u64* xzs, u8* ph, size_t rows, u32 n, int* rank_io,
                   const u64* p_in, u8 p_phase, int keep_result, int phases, int* anticom_out,
                   int* result_out) {
  size_t W = 2 * ((n + 63) / 64);
  Tab t{xzs, ph, W, n};
  bool P = phases != 0;
  std::vector<u64> p(p_in, p_in + W);
  int anticommutes = 0;
  int result = -1;
  if (kind == QCB_STABILIZER || kind == QCB_MIXED_STABILIZER) {
    size_t nr = kind == QCB_STABILIZER ? rows : (size_t)*rank_io;
    for (size_t i = 0; i < nr; i++)
      if (row_comm(p.data(), t.row(i), W)) { anticommutes = (int)i + 1; break; }
    if (anticommutes == 0) {
      if (keep_result || kind == QCB_MIXED_STABILIZER) {
        int rx = 0, rz = 0;
        oracle_canonicalize(xzs, ph, nr, n, phases, &rx, &rz);
        std::vector<u64> g(p);
        u8 gph = p_phase;
        int ok = oracle_generate(g.data(), &gph, xzs, ph, nr, n, phases, nullptr, nullptr);
        if (!ok) { result = -1; anticommutes = rz + 1; }
        else result = gph;
      }
    } else {
      for (size_t i = (size_t)anticommutes; i < nr; i++)
        if (row_comm(p.data(), t.row(i), W)) tab_mul_left(t, i, (size_t)anticommutes - 1, P);
      tab_setrow(t, (size_t)anticommutes - 1, p.data(), p_phase);
    }
    if (kind == QCB_MIXED_STABILIZER) {
      // src/project_trace_reset.jl:310-317
      if (anticommutes == *rank_io + 1 && result == -1) {
        tab_setrow(t, (size_t)*rank_io, p.data(), p_phase);
        *rank_io += 1;
      }
    }
  } else if (kind == QCB_DESTABILIZER) {
    size_t nn = rows / 2, r = nn;
    for (size_t i = 0; i < r; i++)
      if (row_comm(p.data(), t.row(nn + i), W)) { anticommutes = (int)i + 1; break; }
    if (anticommutes == 0) {
      if (nn != n) return QCB_EBADSTRUCT;
      if (keep_result) {
        std::vector<u64> np(W, 0);
        u8 nph = p_phase;
        for (size_t i = 0; i < r; i++)
          if (row_comm(p.data(), t.row(i), W)) {
            u8 e = row_mul_left(np.data(), t.row(nn + i), W, P);
            if (P) nph = (u8)((e + nph + ph[nn + i]) & 3);
          }
        result = nph;
      }
    } else {
      anticomm_update_rows(t, p.data(), r, nn, (size_t)anticommutes, P);
      size_t a = (size_t)anticommutes - 1;
      tab_setrow(t, a, t.row(nn + a), ph[nn + a]);
      tab_setrow(t, nn + a, p.data(), p_phase);
    }
  } else if (kind == QCB_MIXED_DESTABILIZER) {
    size_t nn = rows / 2, r = (size_t)*rank_io;
    for (size_t i = 0; i < r; i++)
      if (row_comm(p.data(), t.row(nn + i), W)) { anticommutes = (int)i + 1; break; }
    if (anticommutes == 0) {
      size_t anticomlog = 0;  // 1-based
      for (size_t i = r; i < nn; i++)
        if (row_comm(p.data(), t.row(i), W)) { anticomlog = i + 1; break; }
      if (anticomlog == 0)
        for (size_t i = nn + r; i < 2 * nn; i++)
          if (row_comm(p.data(), t.row(i), W)) { anticomlog = i + 1; break; }
      if (anticomlog != 0) {
        // 1-based rowswap!(tab, a, b) without phases flag -> phases=true
        if (anticomlog <= nn) {
          tab_rowswap(t, r + nn, anticomlog - 1, true);
          if (nn != r + 1 && anticomlog != r + 1) tab_rowswap(t, r, anticomlog + nn - 1, true);
        } else {
          tab_rowswap(t, r, anticomlog - nn - 1, true);
          tab_rowswap(t, r + nn, anticomlog - 1, true);
        }
        anticomm_update_rows(t, p.data(), r + 1, nn, r + 1, P);
        *rank_io += 1;
        anticommutes = *rank_io;
        tab_setrow(t, r, t.row(nn + r), ph[nn + r]);
        tab_setrow(t, nn + r, p.data(), p_phase);
      } else if (keep_result) {
        std::vector<u64> np(W, 0);
        u8 nph = p_phase;
        for (size_t i = 0; i < r; i++)
          if (row_comm(p.data(), t.row(i), W)) {
            u8 e = row_mul_left(np.data(), t.row(nn + i), W, P);
            if (P) nph = (u8)((e + nph + ph[nn + i]) & 3);
          }
        result = nph;
      }
    } else {
      anticomm_update_rows(t, p.data(), r, nn, (size_t)anticommutes, P);
      size_t a = (size_t)anticommutes - 1;
      tab_setrow(t, a, t.row(nn + a), ph[nn + a]);
      tab_setrow(t, nn + a, p.data(), p_phase);
    }
  }
  *anticom_out = anticommutes;
  *result_out = result;
  return QCB_OK;
}

// evaluate_guesses (src/ecc/decoder_pipeline.jl:172-190): Bool matrices in
// Julia's column-major layout: measured S x nlog, guesses S x k, faults
// nlog x k.  Returns the number of failed samples.
u64 oracle_evaluate_guesses(const u8* measured, const u8* guesses, const u8* faults, u64 S, size_t nlog,
                            size_t k) {
  u64 fails = 0;
  for (u64 i = 0; i < S; i++) {
    for (size_t j = 0; j < nlog; j++) {
      unsigned sum_mod = 0;
      for (size_t c = 0; c < k; c++) sum_mod += (unsigned)(faults[c * nlog + j] & 1u) * (guesses[c * S + i] & 1u);
      sum_mod %= 2;
      if (sum_mod != (unsigned)(measured[j * S + i] & 1u)) {
        fails += 1;
        break;
      }
    }
  }
  return fails;
}

// ---------------------------------------------------------------- states
// The stabilizer view of a state is rows [off, off + rows) of its tableau;
// the Destabilizer kinds pair stabilizer row off + i with destabilizer row i.
struct StateView {
  Tab t;
  size_t off, rows;
  bool destab;
};

static StateView state_view(int kind, u64* xzs, u8* ph, size_t tab_rows, u32 n, int rank) {
  size_t W = 2 * ((n + 63) / 64);
  StateView s{Tab{xzs, ph, W, n}, 0, tab_rows, false};
  if (kind == QCB_MIXED_STABILIZER) s.rows = (size_t)rank;
  if (kind == QCB_DESTABILIZER) { s.off = tab_rows / 2; s.rows = tab_rows / 2; s.destab = true; }
  if (kind == QCB_MIXED_DESTABILIZER) { s.off = tab_rows / 2; s.rows = (size_t)rank; s.destab = true; }
  return s;
}

// rowswap!(state, i, j) (src/QuantumClifford.jl:899-927), 0-based view rows.
static void st_rowswap(StateView& s, size_t i, size_t j, bool P) {
  if (s.destab) tab_rowswap(s.t, i, j, P);
  tab_rowswap(s.t, s.off + i, s.off + j, P);
}

// mul_left!(state, m, i) (src/mul_leftright.jl:195-219): stabilizer m <- i * m;
// the Destabilizer kinds also set destabilizer i <- m * i without phases.
static void st_mul_left(StateView& s, size_t m, size_t i, bool P) {
  if (s.destab) tab_mul_left(s.t, i, m, false);
  tab_mul_left(s.t, s.off + m, s.off + i, P);
}

static bool st_bit(const StateView& s, size_t r, u32 j, int z) {
  return z ? s.t.zbit(s.off + r, j) : s.t.xbit(s.off + r, j);
}

// _canonicalize!(state) (src/canonicalization.jl:95-133) on a state of any kind.
void oracle_canonicalize_state(int kind, u64* xzs, u8* ph, size_t tab_rows, u32 n, int rank, int phases,
                               int* rx_out, int* rz_out) {
  StateView s = state_view(kind, xzs, ph, tab_rows, n, rank);
  bool P = phases != 0;
  size_t i = 0;
  for (int stage = 0; stage < 2; stage++) {
    for (u32 j = 0; j < n; j++) {
      size_t k = s.rows;
      for (size_t ii = i; ii < s.rows; ii++)
        if (st_bit(s, ii, j, stage)) { k = ii; break; }
      if (k == s.rows) continue;
      st_rowswap(s, k, i, P);
      for (size_t m = 0; m < s.rows; m++)
        if (st_bit(s, m, j, stage) && m != i) st_mul_left(s, m, i, P);
      i++;
    }
    if (stage == 0 && rx_out) *rx_out = (int)i;
  }
  if (rz_out) *rz_out = (int)i;
}

// _canonicalize_rref!(state, colindices) (src/canonicalization.jl:153-183).
// cols are 1-based qubits; returns the reference's (1-based) `i`.
int oracle_canonicalize_rref(int kind, u64* xzs, u8* ph, size_t tab_rows, u32 n, int rank,
                             const u32* cols, size_t ncols, int phases) {
  StateView s = state_view(kind, xzs, ph, tab_rows, n, rank);
  bool P = phases != 0;
  long i = (long)s.rows;  // 1-based
  for (size_t c = 0; c < ncols; c++) {
    u32 j = cols[c] - 1;
    for (int z = 0; z < 2; z++) {
      long k = 0;  // findfirst over 1:i
      for (long ii = 1; ii <= i; ii++)
        if (st_bit(s, (size_t)ii - 1, j, z)) { k = ii; break; }
      if (k == 0) continue;
      st_rowswap(s, (size_t)k - 1, (size_t)i - 1, P);
      for (size_t m = 0; m < s.rows; m++)
        if (st_bit(s, m, j, z) && (long)m != i - 1) st_mul_left(s, m, (size_t)i - 1, P);
      i -= 1;
    }
  }
  return (int)i;
}

// permutesystems!(s, perm) (src/linalg.jl:7-17): every row becomes row[perm]
// (new qubit j is old qubit perm[j], 1-based); phases stay.
void oracle_permutesystems(u64* xzs, size_t rows, u32 n, const u32* perm) {
  size_t W = 2 * ((n + 63) / 64), len = W / 2;
  std::vector<u64> old(W);
  for (size_t r = 0; r < rows; r++) {
    u64* row = xzs + r * W;
    std::memcpy(old.data(), row, W * 8);
    for (size_t w = 0; w < W; w++) row[w] = 0;
    for (u32 j = 0; j < n; j++) {
      u32 q = perm[j] - 1;
      row[j >> 6] |= ((old[q >> 6] >> (q & 63)) & 1) << (j & 63);
      row[len + (j >> 6)] |= ((old[len + (q >> 6)] >> (q & 63)) & 1) << (j & 63);
    }
  }
}

// gott_standard_form_indices (src/canonicalization.jl:187-204) on the X
// (half = 0) or Z (half = 1) bits; perm (1-based, length n); returns the rank.
static size_t gott_indices(const u64* xzs, size_t rows, u32 n, int half, size_t skip, u32* perm) {
  size_t W = 2 * ((n + 63) / 64), len = W / 2;
  std::vector<u32> good;
  for (size_t r = skip; r < rows; r++) {
    // unsafe_bitfindnext_(row bits, skip+1) (src/QuantumClifford.jl:960-977)
    long found = -1;
    for (u32 b = (u32)skip; b < 64 * len; b++)
      if ((xzs[r * W + half * len + (b >> 6)] >> (b & 63)) & 1) { found = b; break; }
    if (found < 0) break;
    if (std::find(good.begin(), good.end(), (u32)found + 1) != good.end()) continue;
    good.push_back((u32)found + 1);
  }
  size_t k = 0;
  if (good.empty()) {
    for (u32 j = 1; j <= n; j++) perm[k++] = j;
    return 0;
  }
  for (u32 j = 1; j <= (u32)skip; j++) perm[k++] = j;
  for (u32 g : good) perm[k++] = g;
  for (u32 j = (u32)skip + 1; j <= good.back(); j++)
    if (std::find(good.begin(), good.end(), j) == good.end()) perm[k++] = j;
  for (u32 j = good.back() + 1; j <= n; j++) perm[k++] = j;
  return good.size();
}

// _canonicalize_gott!(stabilizer) (src/canonicalization.jl:223-272) without
// backtracking: returns r, s and the two permutations (1-based, length n).
void oracle_canonicalize_gott(u64* xzs, u8* ph, size_t rows, u32 n, int phases, int* r_out, int* s_out,
                              u32* xperm, u32* zperm) {
  StateView s = state_view(QCB_STABILIZER, xzs, ph, rows, n, 0);
  bool P = phases != 0;
  size_t i = 0;
  for (u32 j = 0; j < n; j++) {
    size_t k = rows;
    for (size_t ii = i; ii < rows; ii++)
      if (st_bit(s, ii, j, 0)) { k = ii; break; }
    if (k == rows) continue;
    st_rowswap(s, k, i, P);
    for (size_t m = 0; m < rows; m++)
      if (st_bit(s, m, j, 0) && m != i) st_mul_left(s, m, i, P);
    i++;
  }
  size_t r = gott_indices(xzs, rows, n, 0, 0, xperm);
  oracle_permutesystems(xzs, rows, n, xperm);
  i = r;
  for (u32 j = (u32)r; j < n; j++) {
    size_t k = rows;
    for (size_t ii = i; ii < rows; ii++)
      if (st_bit(s, ii, j, 1)) { k = ii; break; }
    if (k == rows) continue;
    st_rowswap(s, k, i, P);
    for (size_t m = 0; m < rows; m++)
      if (st_bit(s, m, j, 1) && m != i) st_mul_left(s, m, i, P);
    i++;
  }
  size_t sz = gott_indices(xzs, rows, n, 1, r, zperm);
  oracle_permutesystems(xzs, rows, n, zperm);
  *r_out = (int)r;
  *s_out = (int)sz;
}

// project_cond! (src/project_trace_reset.jl:493-573) behind projectX! /
// projectZ! / projectY! on a MixedDestabilizer: basis 1 = X (condition isZ,
// projector bits (1,0)), 2 = Z (isX, (0,1)), 3 = Y (isXorZ, (1,1)); qubit is
// 1-based.  anticom: 1-based or 0; result: 0..3 or -1 for `nothing`.
void oracle_project_cond(u64* xzs, u8* ph, size_t tab_rows, u32 n, int* rank_io, u32 qubit, int basis,
                         int keep_result, int phases, int* anticom_out, int* result_out) {
  size_t W = 2 * ((n + 63) / 64);
  Tab t{xzs, ph, W, n};
  bool P = phases != 0;
  const u32 q = qubit - 1;
  auto IS = [&](size_t row) -> bool {
    bool x = t.xbit(row, q), z = t.zbit(row, q);
    return basis == 1 ? z : (basis == 2 ? x : (x != z));
  };
  auto set_projector = [&](size_t row) {  // zero!(tab, row); tab[row, qubit] = RESET
    for (size_t w = 0; w < W; w++) t.row(row)[w] = 0;
    t.ph[row] = 0;
    if (basis & 1) t.row(row)[q >> 6] |= 1ull << (q & 63);
    if (basis & 2) t.row(row)[W / 2 + (q >> 6)] |= 1ull << (q & 63);
  };
  // anticomm_update_rows_cond (:480-495), 1-based r and anticommutes
  auto update = [&](size_t r, size_t nn, size_t a) {
    size_t piv = nn + a - 1;
    for (size_t i = r; i < nn; i++)
      if (IS(i)) tab_mul_left(t, i, piv, P);
    for (size_t i = nn + a; i < 2 * nn; i++)
      if (IS(i)) tab_mul_left(t, i, piv, P);
    for (size_t i = 0; i < r; i++)
      if (i != a - 1 && IS(i)) tab_mul_left(t, i, piv, false);
  };
  size_t nn = n, r = (size_t)*rank_io;
  (void)tab_rows;
  int anticommutes = 0, result = -1;
  for (size_t i = 0; i < r; i++)
    if (IS(nn + i)) { anticommutes = (int)i + 1; break; }
  if (anticommutes == 0) {
    size_t anticomlog = 0;
    for (size_t i = r; i < nn; i++)
      if (IS(i)) { anticomlog = i + 1; break; }
    if (anticomlog == 0)
      for (size_t i = nn + r; i < 2 * nn; i++)
        if (IS(i)) { anticomlog = i + 1; break; }
    if (anticomlog != 0) {
      if (anticomlog <= nn) {
        tab_rowswap(t, r + nn, anticomlog - 1, true);
        if (nn != r + 1 && anticomlog != r + 1) tab_rowswap(t, r, anticomlog + nn - 1, true);
      } else {
        tab_rowswap(t, r, anticomlog - nn - 1, true);
        tab_rowswap(t, r + nn, anticomlog - 1, true);
      }
      update(r + 1, nn, r + 1);
      *rank_io += 1;
      anticommutes = *rank_io;
      tab_setrow(t, r, t.row(nn + r), ph[nn + r]);
      set_projector(nn + r);
    } else if (keep_result) {
      std::vector<u64> np(W, 0);
      u8 nph = 0;
      for (size_t i = 0; i < r; i++)
        if (IS(i)) {
          u8 e = row_mul_left(np.data(), t.row(nn + i), W, P);
          if (P) nph = (u8)((e + nph + ph[nn + i]) & 3);
        }
      result = nph;
    }
  } else {
    update(r, nn, (size_t)anticommutes);
    size_t a = (size_t)anticommutes - 1;
    tab_setrow(t, a, t.row(nn + a), ph[nn + a]);
    set_projector(nn + a);
  }
  *anticom_out = anticommutes;
  *result_out = result;
}

// Symbolic gate application with phases (src/symbolic_cliffords.jl:62-74, 293-316).
int oracle_apply_gates(u64* xzs, u8* ph, size_t rows, u32 n, const qcb_op* ops, size_t nops,
                       int phases) {
  size_t W = 2 * ((n + 63) / 64), len = W / 2;
  for (size_t k = 0; k < nops; k++) {
    const qcb_op& op = ops[k];
    if (is1q(op.opcode)) {
      u32 q = op.q1 - 1;
      size_t wi = q >> 6; u64 m = 1ull << (q & 63);
      for (size_t r = 0; r < rows; r++) {
        u64* row = xzs + r * W;
        u64 x = (row[wi] & m) ? 1 : 0, z = (row[len + wi] & m) ? 1 : 0;
        u64 f = gate1(code1(op), x, z) & 1;
        row[wi] = (row[wi] & ~m) | (x & 1 ? m : 0);
        row[len + wi] = (row[len + wi] & ~m) | (z & 1 ? m : 0);
        if (phases && f) ph[r] = (u8)((ph[r] + 2) & 3);
      }
    } else if (is2q(op.opcode)) {
      u32 q1 = op.q1 - 1, q2 = op.q2 - 1;
      size_t w1 = q1 >> 6, w2 = q2 >> 6;
      u64 m1 = 1ull << (q1 & 63), m2 = 1ull << (q2 & 63);
      for (size_t r = 0; r < rows; r++) {
        u64* row = xzs + r * W;
        u64 x1 = (row[w1] & m1) ? 1 : 0, z1 = (row[len + w1] & m1) ? 1 : 0;
        u64 x2 = (row[w2] & m2) ? 1 : 0, z2 = (row[len + w2] & m2) ? 1 : 0;
        u64 f = gate2(op.opcode, x1, z1, x2, z2) & 1;
        row[w1] = (row[w1] & ~m1) | (x1 & 1 ? m1 : 0);
        row[len + w1] = (row[len + w1] & ~m1) | (z1 & 1 ? m1 : 0);
        row[w2] = (row[w2] & ~m2) | (x2 & 1 ? m2 : 0);
        row[len + w2] = (row[len + w2] & ~m2) | (z2 & 1 ? m2 : 0);
        if (phases && f) ph[r] = (u8)((ph[r] + 2) & 3);
      }
    } else {
      return QCB_EUNSUPPORTED;
    }
  }
  return QCB_OK;
}

// Dense apply! (src/dense_cliffords.jl:135-145, apply_row_kernel! :152-169).
// c: 2n rows (images of X_1..X_n then Z_1..Z_n).
void oracle_apply_dense(u64* xzs, u8* ph, size_t rows, u32 n, const u64* c_xzs, const u8* c_ph,
                        int phases) {
  size_t W = 2 * ((n + 63) / 64);
  Tab t{xzs, ph, W, n};
  bool P = phases != 0;
  std::vector<u64> buf(W);
  for (size_t r = 0; r < rows; r++) {
    std::fill(buf.begin(), buf.end(), 0);
    u8 bph = P ? ph[r] : 0;
    for (u32 q = 0; q < n; q++) {
      bool x = t.xbit(r, q), z = t.zbit(r, q);
      if (P && x && z) bph = (u8)(bph - 1);
      if (x) {
        u8 e = row_mul_left(buf.data(), c_xzs + (size_t)q * W, W, P);
        if (P) bph = (u8)((e + bph + c_ph[q]) & 3);
      }
      if (z) {
        u8 e = row_mul_left(buf.data(), c_xzs + (size_t)(q + n) * W, W, P);
        if (P) bph = (u8)((e + bph + c_ph[q + n]) & 3);
      }
    }
    std::memcpy(t.row(r), buf.data(), W * 8);
    // `new_stabrow.phase[]` starts from the row phase only when phases are
    // tracked; s_tab[row] = new_stabrow copies the buffer's phase either way.
    ph[r] = P ? (u8)(bph & 3) : 0;
  }
}

// ------------------------------------------------------------------ frames
// Frame state in the reference layout.
struct Frame {
  u64* xzs; u8* meas; u64 S; u32 nq1; u32 nbits; size_t Wp;
  u64& xw(u32 q, u64 f) const { return xzs[(size_t)(q >> 6) * S + f]; }
  u64& zw(u32 q, u64 f) const { return xzs[(size_t)(Wp / 2 + (q >> 6)) * S + f]; }
};

enum { SRC_MASK = 1, SRC_XOSHIRO = 2 };

struct NoiseFeed {
  int mode;
  // mask mode
  const qcb_event* ev; u64 nev; const u32* reset_planes; u64 words;
  std::vector<std::vector<const qcb_event*>> by_op;  // events grouped by op index
};

static inline bool is_reset(u32 op) { return op == QCB_OP_MRZ || op == QCB_OP_MRX; }
static inline bool is_noise(u32 op) { return op >= QCB_OP_PAULI_NOISE && op <= QCB_OP_DEPOL2; }

// Apply a (noise) Pauli digit to qubit q of frame f: 1=X 2=Z 3=Y.
static inline void frame_flip(Frame& F, u32 q, u64 f, u32 digit) {
  u64 m = 1ull << (q & 63);
  if (digit & 1) F.xw(q, f) ^= m;
  if (digit & 2) F.zw(q, f) ^= m;
}

// One op on frames [f0, f1).  reset_index = index of this op among resets.
// ClassicalXOR (src/pauli_frames.jl:63-72): per frame, record bit `store`
// <- XOR of the listed bits, all read before the store is written.  ops[k] is
// the QCB_OP_XOR header; returns the number of QCB_OP_XOR_BITS ops it used.
static size_t frame_xor(Frame& F, const qcb_op* ops, size_t nops, size_t k, u64 f0, u64 f1) {
  const qcb_op& op = ops[k];
  const u32 n = op.q1;
  const size_t npay = (n + 2) / 3;
  std::vector<u32> bits;
  for (size_t j = 1; j <= npay && k + j < nops; j++)
    for (u32 b : {ops[k + j].q1, ops[k + j].q2, ops[k + j].bit})
      if (b && bits.size() < n) bits.push_back(b - 1);
  u8* dst = F.meas + (size_t)(op.bit - 1) * F.S;
  for (u64 f = f0; f < f1; f++) {
    u8 v = 0;
    for (u32 b : bits) v ^= F.meas[(size_t)b * F.S + f];
    dst[f] = v;
  }
  return npay;
}

static void frame_op(Frame& F, const qcb_op& op, size_t op_index, u64 f0, u64 f1,
                     NoiseFeed& nf, Xoshiro* rng, size_t reset_index) {
  u32 oc = op.opcode;
  if (is1q(oc)) {
    // apply!(f::PauliFrame, op) -> _apply!(..., phases=Val(false))
    u32 q = op.q1 - 1; u64 m = 1ull << (q & 63);
    for (u64 f = f0; f < f1; f++) {
      u64& xw = F.xw(q, f); u64& zw = F.zw(q, f);
      u64 x = (xw & m) ? 1 : 0, z = (zw & m) ? 1 : 0;
      gate1(code1(op), x, z);
      xw = (xw & ~m) | ((x & 1) ? m : 0);
      zw = (zw & ~m) | ((z & 1) ? m : 0);
    }
    return;
  }
  if (is2q(oc)) {
    u32 q1 = op.q1 - 1, q2 = op.q2 - 1;
    u64 m1 = 1ull << (q1 & 63), m2 = 1ull << (q2 & 63);
    for (u64 f = f0; f < f1; f++) {
      u64 x1 = (F.xw(q1, f) & m1) ? 1 : 0, z1 = (F.zw(q1, f) & m1) ? 1 : 0;
      u64 x2 = (F.xw(q2, f) & m2) ? 1 : 0, z2 = (F.zw(q2, f) & m2) ? 1 : 0;
      gate2(oc, x1, z1, x2, z2);
      F.xw(q1, f) = (F.xw(q1, f) & ~m1) | ((x1 & 1) ? m1 : 0);
      F.zw(q1, f) = (F.zw(q1, f) & ~m1) | ((z1 & 1) ? m1 : 0);
      F.xw(q2, f) = (F.xw(q2, f) & ~m2) | ((x2 & 1) ? m2 : 0);
      F.zw(q2, f) = (F.zw(q2, f) & ~m2) | ((z2 & 1) ? m2 : 0);
    }
    return;
  }
  if (oc == QCB_OP_MX || oc == QCB_OP_MRX) {
    // src/pauli_frames.jl:74-83: sHadamard first (and not undone)
    if (oc == QCB_OP_MX && op.bit == 0) return;
    qcb_op h{QCB_OP_H, op.q1, 0, 0, {0, 0, 0}};
    frame_op(F, h, op_index, f0, f1, nf, rng, reset_index);
    qcb_op mz{oc == QCB_OP_MX ? (u32)QCB_OP_MZ : (u32)QCB_OP_MRZ, op.q1, 0, op.bit, {0, 0, 0}};
    frame_op(F, mz, op_index, f0, f1, nf, rng, reset_index);
    return;
  }
  if (oc == QCB_OP_MZ) {
    // src/pauli_frames.jl:85-97
    if (op.bit == 0) return;
    u32 q = op.q1 - 1; u64 m = 1ull << (q & 63);
    u8* col = F.meas + (size_t)(op.bit - 1) * F.S;
    for (u64 f = f0; f < f1; f++) col[f] = (F.xw(q, f) & m) ? 1 : 0;
    return;
  }
  if (oc == QCB_OP_MRZ) {
    // src/pauli_frames.jl:99-116
    u32 q = op.q1 - 1; u64 m = 1ull << (q & 63);
    if (op.bit != 0) {
      u8* col = F.meas + (size_t)(op.bit - 1) * F.S;
      for (u64 f = f0; f < f1; f++) col[f] = (F.xw(q, f) & m) ? 1 : 0;
    }
    for (u64 f = f0; f < f1; f++) {
      F.xw(q, f) &= ~m;
      bool rb;
      if (nf.mode == SRC_MASK)
        rb = nf.reset_planes ? (nf.reset_planes[reset_index * nf.words + (f >> 5)] >> (f & 31)) & 1 : 0;
      else
        rb = rng->next() & 1;
      if (rb) F.zw(q, f) ^= m;
    }
    return;
  }
  if (is_noise(oc)) {
    if (nf.mode == SRC_MASK) {
      if (op_index < nf.by_op.size())
        for (const qcb_event* e : nf.by_op[op_index]) {
          if (e->shot < f0 || e->shot >= f1) continue;
          if (oc == QCB_OP_DEPOL2) {
            frame_flip(F, op.q1 - 1, e->shot, e->pauli & 3);
            frame_flip(F, op.q2 - 1, e->shot, (e->pauli >> 2) & 3);
          } else {
            frame_flip(F, op.q1 - 1, e->shot, e->pauli & 3);
          }
        }
      return;
    }
    if (oc == QCB_OP_PAULI_NOISE) {
      // src/pauli_frames.jl:136-174: X if r<px, Z if r<px+pz, Y if r<px+pz+py
      double px = op.p[0], py = op.p[1], pz = op.p[2];
      u32 q = op.q1 - 1;
      for (u64 f = f0; f < f1; f++) {
        double r = rng->uniform();
        if (r < px) frame_flip(F, q, f, 1);
        else if (r < px + pz) frame_flip(F, q, f, 2);
        else if (r < px + pz + py) frame_flip(F, q, f, 3);
      }
      return;
    }
    // DepolarizationNoise semantics (src/noise.jl:122-132) on each frame.
    int k = oc == QCB_OP_DEPOL2 ? 2 : 1;
    u32 npaulis = 1u << (2 * k);
    for (u64 f = f0; f < f1; f++) {
      if (rng->uniform() >= op.p[0]) continue;
      u32 idx = (u32)(rng->next() % npaulis);
      frame_flip(F, op.q1 - 1, f, idx & 3);
      if (k == 2) frame_flip(F, op.q2 - 1, f, (idx >> 2) & 3);
    }
    return;
  }
}

// pftrajectories(frame, circuit) (src/pauli_frames.jl:234-239), with the
// thread slicing of _pftrajectories (:215-222): nthr = min(threads, S/100).
// mode 1 = mask (events + reset planes), 2 = Xoshiro per slice (seed+slice).
// xzs and meas must already hold the initial frame (see oracle_frame_init_z).
void oracle_pftrajectories(u64* xzs, u8* meas, u64 S, u32 nq1, u32 nbits, const qcb_op* ops,
                           size_t nops, int mode, const qcb_event* events, u64 n_events,
                           const u32* reset_planes, u64 seed, int threads) {
  Frame F{xzs, meas, S, nq1, nbits, 2 * (size_t)((nq1 + 63) / 64)};
  NoiseFeed nf;
  nf.mode = mode; nf.ev = events; nf.nev = n_events; nf.reset_planes = reset_planes;
  nf.words = (S + 31) / 32;
  if (mode == SRC_MASK) {
    nf.by_op.resize(nops);
    for (u64 e = 0; e < n_events; e++)
      if (events[e].op_index < nops) nf.by_op[events[e].op_index].push_back(&events[e]);
  }
  long nthr = std::min<long>(std::max(threads, 1), (long)(S / 100));
  if (nthr < 1) nthr = 1;
  u64 batch = S / nthr;
  auto run = [&](long ti) {
    u64 b = (u64)ti * batch, e = ti == nthr - 1 ? S : (u64)(ti + 1) * batch;
    Xoshiro rng(seed * 0x9E3779B97F4A7C15ull + (u64)ti + 1);
    size_t reset_index = 0;
    for (size_t k = 0; k < nops; k++) {
      if (ops[k].opcode == QCB_OP_XOR) {
        k += frame_xor(F, ops, nops, k, b, e);
        continue;
      }
      frame_op(F, ops[k], k, b, e, nf, &rng, reset_index);
      if (is_reset(ops[k].opcode)) reset_index++;
    }
  };
  if (nthr == 1) { run(0); return; }
  std::vector<std::thread> th;
  for (long ti = 0; ti < nthr; ti++) th.emplace_back(run, ti);
  for (auto& t : th) t.join();
}

// initZ! (src/pauli_frames.jl:47-56).  z_planes (mask mode): [nq1][ceil(S/32)]
// shot-packed bits of each qubit's initial Z; padding bits of the reference
// words are left zero.  z_planes == NULL: Xoshiro words (every Z word, padding
// included, as in the reference).
void oracle_frame_init_z(u64* xzs, u64 S, u32 nq1, const u32* z_planes, u64 seed) {
  size_t Wp = 2 * (size_t)((nq1 + 63) / 64), half = Wp / 2;
  u64 words = (S + 31) / 32;
  if (z_planes) {
    for (size_t w = 0; w < half; w++)
      for (u64 f = 0; f < S; f++) xzs[(half + w) * S + f] = 0;
    for (u32 q = 0; q < nq1; q++)
      for (u64 f = 0; f < S; f++)
        if ((z_planes[(size_t)q * words + (f >> 5)] >> (f & 31)) & 1)
          xzs[(half + (q >> 6)) * S + f] |= 1ull << (q & 63);
  } else {
    Xoshiro rng(seed);
    for (u64 f = 0; f < S; f++)
      for (size_t w = 0; w < half; w++) xzs[(half + w) * S + f] = rng.next();
  }
}

// -------------------------------------------------- Philox-mode replica
// The device's Philox-mode sampling procedure restated on the CPU, so that
// the on-device generator can be checked bit for bit (the reference's own
// streams are checked statistically).  initZ! and reset counters are
// (index, column lo, column hi, tag) with column = global 32-shot word index;
// noise counters are (site, 1024-shot group, block, tag); key = seed.
enum { TAG_INITZ = 0x51A7u, TAG_RESET = 0x5E5Eu, TAG_NOISE = 0x4E01u };

static inline void philox_block(u64 seed, u32 idx, u64 col, u32 tag, u32 out[4]) {
  u32 ctr[4] = {idx, (u32)col, (u32)(col >> 32), tag};
  u32 key[2] = {(u32)seed, (u32)(seed >> 32)};
  oracle_philox4x32_10(ctr, key, out);
}

// Noise sites as the program compiler lays them out, in fixed point:
//  dense sites (p_eff * GROUP > 16) draw one 32-bit word w per shot: PauliNoise
//  X if w < d0, Z if w < d1, Y if w < d2 (units 2^-32); Depolarization an
//  event if w < d2, Pauli index 1 + w*np/d2.
//  sparse sites draw a count word (Binomial(GROUP, p_eff) by inverse CDF
//  against round(P(K<=k) * 2^32)) and one word per event: position w % GROUP,
//  kind word v = w >> 10 (units 2^-22): PauliNoise X if v < s0, Z if v < s1,
//  else Y; Depolarization Pauli index 1 + (v*np >> 22).
static const u32 NOISE_GROUP = 1024, CDF_MAX = 128, KIND_BITS = 22;
struct Site {
  u32 opcode, q1, q2, np;
  bool dense;
  u64 d0, d1, d2, s0, s1;
  std::vector<u32> cdf;
};

static u64 to_fixed(double x, u32 bits) {
  double one = std::ldexp(1.0, (int)bits), f = std::floor(x * one + 0.5);
  if (!(f > 0.0)) return 0;
  return f >= one ? (1ull << bits) : (u64)f;
}

static Site make_site(const qcb_op& op) {
  Site s{op.opcode, op.q1 - 1, op.q2 ? op.q2 - 1 : 0, op.opcode == QCB_OP_DEPOL2 ? 15u : 3u, false, 0, 0, 0, 0, 0, {}};
  double t0, t1, t2, peff;
  if (op.opcode == QCB_OP_PAULI_NOISE) {
    t0 = op.p[0]; t1 = op.p[0] + op.p[2]; t2 = op.p[0] + op.p[2] + op.p[1];
    peff = t2;
  } else {
    double np = op.opcode == QCB_OP_DEPOL2 ? 15.0 : 3.0;
    peff = op.p[0] * np / (np + 1.0);
    t0 = t1 = t2 = peff;
  }
  if (peff > 1.0) peff = 1.0;
  s.dense = peff * NOISE_GROUP > 16.0;
  if (s.dense) {
    s.d0 = to_fixed(t0, 32); s.d1 = to_fixed(t1, 32); s.d2 = to_fixed(std::min(t2, 1.0), 32);
  } else if (peff > 0.0) {
    s.s0 = to_fixed(t0 / peff, KIND_BITS); s.s1 = to_fixed(t1 / peff, KIND_BITS);
    double r = peff / (1.0 - peff), pk = std::pow(1.0 - peff, (double)NOISE_GROUP), cum = pk;
    for (u32 k = 0; k < CDF_MAX; k++) {
      u64 f = to_fixed(cum, 32);
      if (f >> 32) break;
      s.cdf.push_back((u32)f);
      pk = pk * ((double)(NOISE_GROUP - k) * r) / (double)(k + 1);
      cum = cum + pk;
    }
  }
  return s;
}

struct Event { u32 pos, code; };

// Events of one site on one group of NOISE_GROUP shots: word i of Philox block
// (site, group, i/4, TAG_NOISE) lane i%4.
static void site_group_events(const Site& s, u32 site, u64 group, u64 seed, std::vector<Event>& out) {
  u32 key[2] = {(u32)seed, (u32)(seed >> 32)};
  u32 o[4];
  if (s.dense) {
    for (u32 blk = 0; blk < NOISE_GROUP / 4; blk++) {
      u32 ctr[4] = {site, (u32)group, blk, TAG_NOISE};
      oracle_philox4x32_10(ctr, key, o);
      for (u32 j = 0; j < 4; j++) {
        u64 w = o[j];
        u32 code = 0;
        if (s.opcode == QCB_OP_PAULI_NOISE) code = w < s.d0 ? 1 : w < s.d1 ? 2 : w < s.d2 ? 3 : 0;
        else if (w < s.d2) code = 1 + (u32)(w * s.np / s.d2);
        if (code) out.push_back({blk * 4 + j, code});
      }
    }
    return;
  }
  if (s.cdf.empty()) return;
  u32 ctr0[4] = {site, (u32)group, 0u, TAG_NOISE};
  oracle_philox4x32_10(ctr0, key, o);
  u32 k = 0;
  while (k < s.cdf.size() && o[0] >= s.cdf[k]) k++;
  auto word = [&](u32 i) {
    u32 ctr[4] = {site, (u32)group, i >> 2, TAG_NOISE}, b[4];
    oracle_philox4x32_10(ctr, key, b);
    return b[i & 3];
  };
  // event e starts from word 1+e; in order, an event whose position repeats
  // an earlier event's takes the next unused word (k+1, k+2, ...), at most
  // 64 times, after which the last draw is kept
  std::vector<bool> used(NOISE_GROUP, false);
  u32 next = k + 1;
  for (u32 e = 0; e < k; e++) {
    u32 w = word(1 + e);
    for (u32 r = 0; r < 64 && used[w % NOISE_GROUP]; r++) w = word(next++);
    used[w % NOISE_GROUP] = true;
    u32 v = w >> 10, code;
    if (s.opcode == QCB_OP_PAULI_NOISE) code = v < s.s0 ? 1 : v < s.s1 ? 2 : 3;
    else code = 1 + ((v * s.np) >> KIND_BITS);
    out.push_back({w % NOISE_GROUP, code});
  }
}

// Runs the op list on the frame in Philox mode exactly as the device does.
// Frame x/z must be preset (x=0 and Z from oracle_philox_init_z for a fresh
// frame).  shot_offset: global shot of frame 0 (multiple of 1024).
void oracle_pftrajectories_philox(u64* xzs, u8* meas, u64 S, u32 nq1, u32 nbits,
                                  const qcb_op* ops, size_t nops, u64 seed, u64 shot_offset) {
  Frame F{xzs, meas, S, nq1, nbits, 2 * (size_t)((nq1 + 63) / 64)};
  std::vector<Site> sites;
  std::vector<long> site_of_op(nops, -1);
  for (size_t k = 0; k < nops; k++) {
    if (!is_noise(ops[k].opcode)) continue;
    site_of_op[k] = (long)sites.size();
    sites.push_back(make_site(ops[k]));
  }
  const u64 words = (S + 31) / 32, col0 = shot_offset / 32;
  for (u64 g0 = 0; g0 < words; g0 += 32) {  // groups of 32 columns = 1024 shots
    const u64 group = (col0 + g0) / 32;
    std::vector<std::vector<Event>> ev(sites.size());
    for (u32 s = 0; s < (u32)sites.size(); s++) site_group_events(sites[s], s, group, seed, ev[s]);
    for (u64 w = g0; w < std::min<u64>(words, g0 + 32); w++) {
      const u64 col = col0 + w;
      const u64 f0 = w * 32, f1 = std::min<u64>(S, f0 + 32);
      size_t reset_index = 0;
      u32 rcache[4];
      u32 rblock = 0xFFFFFFFFu;
      for (size_t k = 0; k < nops; k++) {
        const qcb_op& op = ops[k];
        const u32 oc = op.opcode;
        if (oc == QCB_OP_XOR) {
          k += frame_xor(F, ops, nops, k, f0, f1);
          continue;
        }
        if (is_noise(oc)) {
          const Site& st = sites[(size_t)site_of_op[k]];
          for (const Event& e : ev[(size_t)site_of_op[k]]) {
            const u64 f = (g0 + (e.pos >> 5)) * 32 + (e.pos & 31);
            if (f < f0 || f >= f1) continue;
            if (st.opcode == QCB_OP_DEPOL2) {
              frame_flip(F, st.q1, f, e.code & 3);
              frame_flip(F, st.q2, f, (e.code >> 2) & 3);
            } else {
              frame_flip(F, st.q1, f, e.code & 3);
            }
          }
          continue;
        }
        if (oc == QCB_OP_MRZ || oc == QCB_OP_MRX) {
          const u32 q = op.q1 - 1;
          const u64 m = 1ull << (q & 63);
          if (oc == QCB_OP_MRX) {
            for (u64 f = f0; f < f1; f++) {
              const u64 x = (F.xw(q, f) & m) ? 1 : 0, z = (F.zw(q, f) & m) ? 1 : 0;
              F.xw(q, f) = (F.xw(q, f) & ~m) | (z ? m : 0);
              F.zw(q, f) = (F.zw(q, f) & ~m) | (x ? m : 0);
            }
          }
          if (rblock != (u32)(reset_index >> 2)) {
            rblock = (u32)(reset_index >> 2);
            philox_block(seed, rblock, col, TAG_RESET, rcache);
          }
          const u32 rb = rcache[reset_index & 3];
          if (op.bit != 0) {
            u8* c = F.meas + (size_t)(op.bit - 1) * F.S;
            for (u64 f = f0; f < f1; f++) c[f] = (F.xw(q, f) & m) ? 1 : 0;
          }
          for (u64 f = f0; f < f1; f++) {
            F.xw(q, f) &= ~m;
            if ((rb >> (f - f0)) & 1) F.zw(q, f) ^= m;
          }
          reset_index++;
          continue;
        }
        NoiseFeed nf;
        nf.mode = SRC_MASK;
        frame_op(F, op, k, f0, f1, nf, nullptr, 0);
      }
    }
  }
}

// Philox initZ!: z bit of qubit q, shot s = bit (s&31) of
// philox(q>>2, column, TAG_INITZ)[q&3]; x bits cleared.
void oracle_philox_init_z(u64* xzs, u64 S, u32 nq1, u64 seed, u64 shot_offset) {
  size_t Wp = 2 * (size_t)((nq1 + 63) / 64), half = Wp / 2;
  std::memset(xzs, 0, Wp * S * 8);
  u64 words = (S + 31) / 32, col0 = shot_offset / 32;
  for (u64 w = 0; w < words; w++) {
    u32 o[4];
    for (u32 q = 0; q < nq1; q++) {
      if ((q & 3) == 0) philox_block(seed, q >> 2, col0 + w, TAG_INITZ, o);
      u32 bits = o[q & 3];
      for (u32 l = 0; l < 32; l++) {
        u64 f = w * 32 + l;
        if (f >= S) break;
        if ((bits >> l) & 1) xzs[(half + (q >> 6)) * S + f] |= 1ull << (q & 63);
      }
    }
  }
}

}  // extern "C"
