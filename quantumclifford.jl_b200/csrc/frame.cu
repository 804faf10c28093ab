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
// Noise (Philox mode).  Counter-based streams (key = seed): initZ! and reset
// draws per (index, shot column); noise per (site, group of 1024 shots), where
// one word gives the group's Binomial event count and one word per event its
// shot and kind, in integer fixed point (sample_site_group).  The sites of a
// FLUSH record are sampled there, as (site, group) tasks spread over the
// whole CTA, and flipped into the tile with shared-memory atomics.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <unordered_map>

#include "qcb_internal.h"

namespace qcb {

struct WalkArgs {
  const uint4* prog;        // windowed stream (win_words words per window)
  uint32_t nwin;            // windows in the stream
  uint32_t win_words;       // words per window (the program's)
  uint32_t* planes;
  uint32_t* rec;            // record row b at rec + b * rec_pitch (column 0 of this frame)
  uint64_t pitch;
  uint64_t rec_pitch;
  uint64_t ncols;
  const uint32_t* slot_qubit;
  const uint32_t* slot_swap;
  uint32_t nslots;
  uint32_t nq1;
  uint32_t fresh;           // 1: start from x = 0, z = Philox initZ!
  uint32_t tile;            // shot columns per tile (multiple of 32)
  const uint32_t* qubit_slot;
  uint32_t qubit_slot_len;
  uint64_t seed;
  uint64_t col0;            // global column index of column 0
  const NoiseClass* classes;
  const uint32_t* cdf;      // Binomial count tables of the sparse classes
  double pmax;
  int32_t* err;             // set to QCB_ETIMEOUT when a staging wait gives up
  // mask mode
  const uint64_t* ev_off;
  const uint64_t* ev_data;  // (trial << 8) | code, sorted per column
  const uint32_t* reset_planes;
  uint64_t reset_pitch;
  // test knob: window index (of each CTA's sequence) that is never staged, so
  // the walker's bounded wait runs out (0: none)
  uint64_t withhold;
  // pre-sampled noise (null: the walk draws every (site, group) itself):
  // bucket (group g, flush part j) holds pre_cnt[g * pre_nparts + j] events
  // at pre_buf + g * pre_capg + pre_capoff[j] (at most pre_capoff[j + 1] -
  // pre_capoff[j]; a fuller bucket is drawn in the walk); g counts groups
  // from the run's first column
  const uint32_t* pre_buf;
  const uint32_t* pre_cnt;
  const uint32_t* pre_capoff;
  uint32_t pre_nparts;
  uint32_t pre_capg;
};

// Bit-sliced single-qubit gate (src/symbolic_cliffords.jl:105-118); frames
// track no phase (src/pauli_frames.jl:58-61).
__device__ __forceinline__ void gate1_xz(uint32_t op, uint32_t& x, uint32_t& z) {
  const uint32_t X = x, Z = z;
  if ((op & 0xFFu) == QCB_OP_SQO) {  // SingleQubitOperator, flags in bits 8..13
    const uint32_t xx = 0u - ((op >> 8) & 1u), xz = 0u - ((op >> 9) & 1u);
    const uint32_t zx = 0u - ((op >> 10) & 1u), zz = 0u - ((op >> 11) & 1u);
    x = (X & xx) ^ (Z & zx);
    z = (X & xz) ^ (Z & zz);
    return;
  }
  switch (op) {
    case QCB_OP_H: case QCB_OP_SQRTY: case QCB_OP_INVSQRTY: x = Z; z = X; break;
    case QCB_OP_HXY: case QCB_OP_S: case QCB_OP_SDAG: z = X ^ Z; break;
    case QCB_OP_HYZ: case QCB_OP_SQRTX: case QCB_OP_INVSQRTX: x = X ^ Z; break;
    case QCB_OP_CXYZ: x = X ^ Z; z = X; break;
    case QCB_OP_CZYX: x = Z; z = X ^ Z; break;
    default: break;  // I, X, Y, Z: no change to the frame bits
  }
}

// Bit-sliced two-qubit gate maps (src/symbolic_cliffords.jl:358-395).
__device__ __forceinline__ void gate2_xz(uint32_t op, uint32_t& x1, uint32_t& z1, uint32_t& x2,
                                         uint32_t& z2) {
  const uint32_t a = x1, b = z1, c = x2, d = z2;
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
    case QCB_OP_SWAPCX: x1 = c; z1 = d ^ b; x2 = c ^ a; z2 = b; break;
    case QCB_OP_INVSWAPCX: case QCB_OP_CXSWAP: x1 = c ^ a; z1 = d; x2 = a; z2 = d ^ b; break;
    case QCB_OP_ISWAP: case QCB_OP_INVISWAP: x1 = c; z1 = a ^ d ^ c; x2 = a; z2 = a ^ c ^ b; break;
    case QCB_OP_CZSWAP: x1 = c; z1 = d ^ a; x2 = a; z2 = c ^ b; break;
    case QCB_OP_ZCRY: case QCB_OP_INVZCRY: z1 = a ^ b ^ c ^ d; x2 = a ^ c; z2 = a ^ d; break;
    case QCB_OP_SQRTZZ: case QCB_OP_INVSQRTZZ: z1 = a ^ c ^ b; z2 = a ^ d ^ c; break;
    case QCB_OP_SQRTXX: case QCB_OP_INVSQRTXX: x1 = b ^ d ^ a; x2 = b ^ c ^ d; break;
    case QCB_OP_SQRTYY: case QCB_OP_INVSQRTYY:
      x1 = b ^ c ^ d; z1 = a ^ d ^ c; x2 = a ^ b ^ d; z2 = a ^ c ^ b; break;
    default: break;
  }
}

// The frame tile.  SMEM: plane p of tile column cl at sm[p*T + cl] (T even).
// Global: plane p maps to frame plane pmap[p] (a shared-memory table).
template <bool SMEM>
struct Tile {
  uint32_t* sm;
  uint32_t* planes;
  const uint32_t* pmap;
  uint64_t pitch;
  uint32_t T;
  // word of plane p at tile column cl (frame column cg)
  __device__ __forceinline__ uint32_t* at32(uint32_t p, uint32_t cl, uint64_t cg) const {
    if (SMEM) return sm + p * T + cl;
    return planes + (uint64_t)pmap[p] * pitch + cg;
  }
  // the two words of plane p at the even tile column cw (frame column cg)
  __device__ __forceinline__ uint2* at2(uint32_t p, uint32_t cw, uint64_t cg) const {
    return (uint2*)at32(p, cw, cg);
  }
};

__device__ __forceinline__ uint32_t sel4(const uint32_t o[4], uint32_t i) {
  const uint32_t a = (i & 1) ? o[1] : o[0];
  const uint32_t b = (i & 1) ? o[3] : o[2];
  return (i & 2) ? b : a;
}

// ---------------------------------------------------------------- staging
// The program is staged window by window into two shared-memory buffers with
// bulk copies (cp.async.bulk, completion on an mbarrier), one window ahead of
// the walk.  Waits are bounded: on expiry the kernel records QCB_ETIMEOUT.
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void stage_window(uint32_t* dst, const uint4* src, uint32_t bytes, uint64_t* bar) {
  const uint32_t b = smem_addr(bar);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(b)
      : "memory");
}

// Bounded wait for the phase `parity` of an mbarrier: each poll suspends at
// most WAIT_POLL_NS, and the wait gives up after WAIT_LIMIT_NS of the global
// timer (or 2^24 polls, whichever comes first).  Returns false when it gave up.
constexpr uint32_t WAIT_POLL_NS = 2000;
constexpr uint64_t WAIT_LIMIT_NS = 1000000000ull;  // one second

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t b = smem_addr(bar);
  uint64_t t0 = 0;
  for (uint32_t it = 0; it < (1u << 24); it++) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(b), "r"(parity), "r"(WAIT_POLL_NS)
        : "memory");
    if (ok) return true;
    const uint64_t now = global_ns();
    if (it == 0) t0 = now;
    else if (now - t0 > WAIT_LIMIT_NS) return false;
  }
  return false;
}

// ---------------------------------------------------------------- noise
// Event codes: bit 0 flips x of the site's first qubit, bit 1 its z, bits 2
// and 3 the same for the second qubit; 0 is no event.  PauliNoise gives X = 1,
// Z = 2, Y = 3; DepolarizationNoise a uniform non-identity Pauli index.
// Dense draw: one 32-bit word per shot (thresholds in units of 2^-32).
__device__ __forceinline__ uint32_t dense_code(uint32_t kind, const NoiseClass& c, uint32_t w) {
  if (kind == QCB_OP_PAULI_NOISE) return w < c.thr0 ? 1u : w < c.thr1 ? 2u : w < c.thr2 ? 3u : 0u;
  if (w >= c.thr2) return 0u;
  return 1u + (uint32_t)(((uint64_t)w * c.np) / c.thr2);
}

// Sparse event: the kind of an event that happens, from a 22-bit word v.
__device__ __forceinline__ uint32_t sparse_code(uint32_t kind, const NoiseClass& c, uint32_t v) {
  if (kind == QCB_OP_PAULI_NOISE) return v < c.thr0 ? 1u : v < c.thr1 ? 2u : 3u;
  return 1u + ((v * c.np) >> NOISE_KIND_BITS);
}

// Flip the event's Pauli into the tile at group shot `pos`; lc0 is the tile
// column of the group's first column (a group may straddle tiles: columns
// outside [0, T) belong to a neighbouring tile, which draws the same events).
// e = (site, kind | class<<8, x_a | z_a<<16, x_b | z_b<<16).
template <bool SMEM>
__device__ __forceinline__ void apply_code(const Tile<SMEM>& F, const uint4& e, uint32_t code, int32_t lc0,
                                           uint32_t pos, uint64_t c0, uint64_t ncols) {
  const int32_t lc = lc0 + (int32_t)(pos >> 5);
  if (lc < 0 || lc >= (int32_t)F.T) return;
  const uint32_t cl = (uint32_t)lc;
  const uint64_t cg = c0 + cl;
  if (cg >= ncols) return;
  const uint32_t bit = 1u << (pos & 31);
  if (code & 1) atomicXor(F.at32(e.z & 0xFFFFu, cl, cg), bit);
  if (code & 2) atomicXor(F.at32(e.z >> 16, cl, cg), bit);
  if ((e.y & 0xFFu) == QCB_OP_DEPOL2) {
    if (code & 4) atomicXor(F.at32(e.w & 0xFFFFu, cl, cg), bit);
    if (code & 8) atomicXor(F.at32(e.w >> 16, cl, cg), bit);
  }
}

// Word i of the noise stream of (site, group G): lane i % 4 of Philox block
// (site, G, i / 4, TAG_NOISE).
__device__ __forceinline__ uint32_t noise_word(uint32_t site, uint32_t glo, uint32_t i, uint32_t k0,
                                               uint32_t k1) {
  uint32_t o[4];
  philox4x32_10(site, glo, i >> 2, TAG_NOISE, k0, k1, o);
  return sel4(o, i & 3);
}

// Events with at most this many per (site, group) stay in registers (the
// rest take the 1024-bit bitmap path, slow enough that a warp with one such
// lane pays for it: d=11 launch 0.94 / 0.84 / 0.668 / 0.674 ms at 3 / 4 / 6 / 8).
constexpr uint32_t NOISE_KREG = 6;
// Redraws of one event's position before its last draw is kept (a collision
// has probability below k/NOISE_GROUP per draw, so the cap is never reached
// in practice; it only bounds the loop).
constexpr uint32_t NOISE_REDRAWS = 64;

// The events of one noise site on one group of NOISE_GROUP shots (group G of
// the run, = 32 consecutive shot columns), from the words of noise_word.
//  sparse: word 0 gives the event count k ~ Binomial(NOISE_GROUP, p_eff) by
//          inverse CDF against the class's fixed-point table.  Event e starts
//          from word 1 + e: position w & (NOISE_GROUP-1), kind from w >> 10.
//          Then, for e = 1, 2, ... in order, while event e's position equals
//          that of an earlier event, its word is replaced by the next unused
//          word k+1, k+2, ...  This is sequential rejection sampling, so given
//          k the positions are a uniform k-subset and the kinds are
//          independent: every shot gets an event independently with
//          probability p_eff, as the reference's per-frame draws.
//  dense:  word j is the per-shot draw of shot j.
// Sparse classes (see sample_site_group): the event count k of (site, group)
// from Philox block 0, whose words 1..3 `o` keeps for the first events.
__device__ __forceinline__ uint32_t sparse_count(const NoiseClass& c, const uint32_t* cdf, uint32_t site,
                                                 uint32_t glo, uint32_t k0, uint32_t k1, uint32_t o[4]) {
  if (!c.cdf_len) return 0;
  philox4x32_10(site, glo, 0u, TAG_NOISE, k0, k1, o);
  // k = number of table entries <= word 0 (the table is non-decreasing, so
  // this is the inverse CDF), four entries per 16-byte read: one read for
  // counts below 4
  const uint4* tb = (const uint4*)(cdf + c.cdf_off);
  uint32_t k = 0;
  for (uint32_t b = 0; b < c.cdf_len; b += 4) {
    const uint4 t = __ldg(tb + (b >> 2));
    const uint32_t lim = c.cdf_len - b;
    const uint32_t m = (uint32_t)(o[0] >= t.x) + (uint32_t)(lim > 1 && o[0] >= t.y) +
                       (uint32_t)(lim > 2 && o[0] >= t.z) + (uint32_t)(lim > 3 && o[0] >= t.w);
    k += m;
    if (m < 4) break;
  }
  return k;
}

// The k events of (site, group) as emit(position, code): event e from word
// 1 + e, a position already taken redrawn from the next unused word.  Up to
// KREG events are kept in registers, more in a bitmap; both are the same
// sequential procedure, so KREG changes the cost and not the events.
template <uint32_t KREG = NOISE_KREG, class Emit>
__device__ __forceinline__ void sparse_emit(const NoiseClass& c, uint32_t kind, uint32_t site, uint32_t glo,
                                            uint32_t k0, uint32_t k1, uint32_t k, uint32_t o[4], Emit emit) {
  constexpr uint32_t PMASK = NOISE_GROUP - 1;
  uint32_t next = k + 1;  // next unused word
  if (k <= KREG) {
    uint32_t w[KREG];
#pragma unroll
    for (uint32_t ev = 0; ev < KREG; ev++) {
      if (ev < k) {
        if (((ev + 1) & 3) == 0) philox4x32_10(site, glo, (ev + 1) >> 2, TAG_NOISE, k0, k1, o);
        w[ev] = o[(ev + 1) & 3];
      }
    }
#pragma unroll
    for (uint32_t ev = 1; ev < KREG; ev++) {
      if (ev < k) {
        for (uint32_t r = 0; r < NOISE_REDRAWS; r++) {
          bool dup = false;
#pragma unroll
          for (uint32_t j = 0; j < ev; j++) dup |= ((w[ev] ^ w[j]) & PMASK) == 0;
          if (!dup) break;
          w[ev] = noise_word(site, glo, next++, k0, k1);
        }
      }
    }
#pragma unroll
    for (uint32_t ev = 0; ev < KREG; ev++)
      if (ev < k) emit(w[ev] & PMASK, sparse_code(kind, c, w[ev] >> 10));
    return;
  }
  uint32_t bm[NOISE_GROUP / 32];  // positions taken so far
  for (uint32_t i = 0; i < NOISE_GROUP / 32; i++) bm[i] = 0;
  uint32_t blk = 0;  // o holds Philox block blk of the stream (block 0: the count word and words 1..3)
  for (uint32_t ev = 0; ev < k; ev++) {
    if (((1 + ev) >> 2) != blk) {
      blk = (1 + ev) >> 2;
      philox4x32_10(site, glo, blk, TAG_NOISE, k0, k1, o);
    }
    uint32_t wv = sel4(o, (1 + ev) & 3);  // word 1 + ev, one block per four events
    for (uint32_t r = 0; r < NOISE_REDRAWS && ((bm[(wv & PMASK) >> 5] >> (wv & 31)) & 1u); r++)
      wv = noise_word(site, glo, next++, k0, k1);
    bm[(wv & PMASK) >> 5] |= 1u << (wv & 31);
    emit(wv & PMASK, sparse_code(kind, c, wv >> 10));
  }
}

template <bool SMEM>
__device__ __forceinline__ void sample_site_group(const WalkArgs& a, const Tile<SMEM>& F, const uint4& e,
                                                  uint64_t G, int32_t lc0, uint64_t c0) {
  const uint32_t site = e.x, kind = e.y & 0xFFu;
  const NoiseClass c = a.classes[e.y >> 8];
  const uint32_t k0 = (uint32_t)a.seed, k1 = (uint32_t)(a.seed >> 32);
  const uint32_t glo = (uint32_t)G;
  uint32_t o[4];
  if (c.dense) {
    for (uint32_t blk = 0; blk < NOISE_GROUP / 4; blk++) {
      philox4x32_10(site, glo, blk, TAG_NOISE, k0, k1, o);
#pragma unroll
      for (uint32_t j = 0; j < 4; j++) {
        const uint32_t code = dense_code(kind, c, o[j]);
        if (code) apply_code<SMEM>(F, e, code, lc0, blk * 4 + j, c0, a.ncols);
      }
    }
    return;
  }
  const uint32_t k = sparse_count(c, a.cdf, site, glo, k0, k1, o);
  if (k == 0) return;
  sparse_emit(c, kind, site, glo, k0, k1, k, o,
              [&](uint32_t pos, uint32_t code) { apply_code<SMEM>(F, e, code, lc0, pos, c0, a.ncols); });
}

// ---------------------------------------------------------------- pre-sampling
// Every sparse (site, group) of a Philox run drawn before the walk, in a
// grid of its own (no CTA barriers, full occupancy): thread (entry, group)
// draws the site's events on the group exactly as sample_site_group would and
// appends them to the bucket (group, flush part) as words
// (entry index << 16 | code << 10 | position), the slot from an atomic on the
// bucket's count.  Event order inside a bucket does not matter (flips are
// XORs).  A bucket whose count ends above its capacity keeps only part of its
// events; the walk then draws that bucket itself.
struct PresampleArgs {
  const uint4* ent;         // (site, kind | class << 8, part j, entry index i)
  uint32_t nent;
  uint32_t nparts;
  uint64_t g0;              // global group index of the run's first group
  uint64_t ngroups;
  const NoiseClass* classes;
  const uint32_t* cdf;
  uint64_t seed;
  uint32_t* cnt;            // [ngroups][nparts], zero before the launch
  uint32_t* buf;            // [ngroups][capg]
  const uint32_t* capoff;   // [nparts + 1]
  uint32_t capg;
  uint32_t force_overflow;  // test knob: every non-empty bucket reports more than its capacity
};

__global__ void __launch_bounds__(256) presample_kernel(const PresampleArgs p) {
  // the walker that reads these buckets is a programmatic dependent: let it
  // launch once every sampler CTA is resident, so that its CTAs take the SMs
  // of the sampler's last wave as they free up (it waits before its first read)
  asm volatile("griddepcontrol.launch_dependents;");
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x, lane = threadIdx.x & 31;
  const bool valid = e < p.nent;
  const uint4 pe = valid ? p.ent[e] : make_uint4(0u, 0u, 0xFFFFFFFFu, 0u);
  NoiseClass c{};
  if (valid) c = p.classes[pe.y >> 8];
  const uint32_t kind = pe.y & 0xFFu, j = pe.z;
  const uint32_t k0 = (uint32_t)p.seed, k1 = (uint32_t)(p.seed >> 32);
  const uint32_t off = valid ? p.capoff[j] : 0u, cap = valid ? p.capoff[j + 1] - off : 0u;
  // The entries are sorted by part, so the lanes of one part form a run
  // [first, last]: its events take one atomic on the bucket count (by the
  // run's last lane) and consecutive slots.
  const uint32_t peers = __match_any_sync(0xFFFFFFFFu, j);
  const uint32_t first = __ffs(peers) - 1, last = 31 - __clz(peers);
  const uint32_t tag = pe.w << 16;
  for (uint64_t g = blockIdx.y; g < p.ngroups; g += gridDim.y) {
    const uint32_t glo = (uint32_t)(p.g0 + g);
    uint32_t o[4];
    const uint32_t k = valid ? sparse_count(c, p.cdf, pe.x, glo, k0, k1, o) : 0u;
    uint32_t inc = k;  // inclusive prefix of k over the run
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
      const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, inc, d);
      if (lane >= first + d) inc += v;
    }
    uint32_t base = 0;
    if (lane == last && inc) base = atomicAdd(p.cnt + g * p.nparts + j, inc + (p.force_overflow ? cap + 1 : 0u));
    base = __shfl_sync(0xFFFFFFFFu, base, last);
    if (k == 0) continue;
    uint32_t* bk = p.buf + g * p.capg + off;
    uint32_t t = base + inc - k;
    auto put = [&](uint32_t pos, uint32_t code) {
      if (t < cap) bk[t] = tag | (code << 10) | pos;
      t++;
    };
    // most counts are below 4 (block 0's words 1..3): a short path for them
    if (k <= 3) sparse_emit<3>(c, kind, pe.x, glo, k0, k1, k, o, put);
    else sparse_emit<NOISE_KREG>(c, kind, pe.x, glo, k0, k1, k, o, put);
  }
}

// ---------------------------------------------------------------- walker
__device__ __forceinline__ uint2 xor2(uint2 a, uint2 b) { return make_uint2(a.x ^ b.x, a.y ^ b.y); }

// One tile of T shot columns (T even; T x 32 shots) walked through the whole
// program by one CTA.  Thread (rr, cp) = (tid / TP, tid % TP), TP = T / 2,
// handles the column pair (2cp, 2cp + 1) -- one 64-bit shared-memory word per
// plane, so each op's operand decode and address arithmetic serve two columns
// -- and every R-th op of a segment; a warp covers consecutive pairs of one
// op (broadcast operand reads from the staged window).  One barrier per
// record orders the records.  The program arrives window by window in the
// two staging buffers (window kwin in buffer kwin & 1); after each window
// thread 0 calls issue(kwin + 2) for the window two ahead.  Returns false
// when a staging wait gave up (the job's status word then holds
// QCB_ETIMEOUT).
template <bool SMEM, bool PHILOX, bool PRE, class Issue>
__device__ __forceinline__ bool walk_tile(const WalkArgs& a, uint32_t* sm, uint32_t* win0, uint32_t* win1,
                                          uint64_t* bars, uint64_t& kwin, Issue& issue, uint64_t tile) {
  const uint32_t tid = threadIdx.x, T = a.tile, TP = T / 2, R = blockDim.x / TP;
  const uint32_t cp = tid % TP, rr = tid / TP, cw = 2 * cp;  // cw: tile column of the pair
  const uint32_t k0 = (uint32_t)a.seed, k1 = (uint32_t)(a.seed >> 32);
  const uint64_t pitch = a.pitch, rpitch = a.rec_pitch;
  const uint64_t c0 = tile * T, cg = c0 + cw;  // the pair's first column in the frame
  const bool act = rr < R && cg < a.ncols;
  const bool two = cg + 1 < a.ncols;          // its second column exists
  const uint64_t col = a.col0 + cg, col1 = col + 1;
  const uint32_t clo = (uint32_t)col, chi = (uint32_t)(col >> 32);
  const uint32_t clo1 = (uint32_t)col1, chi1 = (uint32_t)(col1 >> 32);
  const Tile<SMEM> F{sm, a.planes, sm, pitch, T};

  // ---- initial frame
  if (a.fresh) {
    for (uint32_t qb = rr; qb * 4 < a.nq1; qb += R) {
      if (!act) break;
      uint32_t o[4], u[4];
      philox4x32_10(qb, clo, chi, TAG_INITZ, k0, k1, o);
      philox4x32_10(qb, clo1, chi1, TAG_INITZ, k0, k1, u);
#pragma unroll
      for (uint32_t j = 0; j < 4; j++) {
        const uint32_t q = qb * 4 + j;
        if (q >= a.nq1) break;
        const uint32_t s = (SMEM && q < a.qubit_slot_len) ? __ldg(a.qubit_slot + q) : BIT_NONE;
        if (SMEM && s != BIT_NONE) {
          *F.at2(2 * s, cw, cg) = make_uint2(0u, 0u);
          *F.at2(2 * s + 1, cw, cg) = make_uint2(o[j], u[j]);
        } else {
          *(uint2*)(a.planes + (uint64_t)(2 * q) * pitch + cg) = make_uint2(0u, 0u);
          *(uint2*)(a.planes + (uint64_t)(2 * q + 1) * pitch + cg) = make_uint2(o[j], u[j]);
        }
      }
    }
  } else if (SMEM) {
    for (uint32_t s = rr; s < a.nslots; s += R) {
      if (!act) break;
      const uint32_t q = __ldg(a.slot_qubit + s);
      *F.at2(2 * s, cw, cg) = *(const uint2*)(a.planes + (uint64_t)(2 * q) * pitch + cg);
      *F.at2(2 * s + 1, cw, cg) = *(const uint2*)(a.planes + (uint64_t)(2 * q + 1) * pitch + cg);
    }
  }
  // mask mode: the events of the pair's columns, [ep[h], ep[h + 1]) for column h
  uint64_t ep[3] = {0, 0, 0};
  if (!PHILOX && rr == 0 && act) {
    ep[0] = a.ev_off[cg];
    ep[1] = a.ev_off[cg + 1];
    ep[2] = two ? a.ev_off[cg + 2] : ep[1];
  }

  // ---- pre-sampled noise: thread (pgl, pl) takes events pl, pl + pS, ... of
  // the buckets of its group G0 + pgl of the tile; the count and the first
  // two events of the next flush part are loaded one part ahead (issued at a
  // flush, they arrive while the following records run)
  const uint64_t pG0 = (a.col0 + c0) / 32;
  const uint32_t png = (uint32_t)((a.col0 + min(c0 + T, a.ncols) - 1) / 32 - pG0 + 1);
  const uint32_t pS = blockDim.x / png, pgl = tid / pS, pl = tid - pgl * pS;
  const bool pre = PRE && PHILOX && a.pre_buf != nullptr && pgl < png;
  const uint32_t* pbase = pre ? a.pre_buf + (pG0 + pgl - a.col0 / 32) * a.pre_capg : nullptr;
  const uint32_t* pcnt = pre ? a.pre_cnt + (pG0 + pgl - a.col0 / 32) * a.pre_nparts : nullptr;
  uint32_t pf_tot = 0, pf_e0 = 0, pf_e1 = 0;
  auto prefetch = [&](uint32_t jn, uint32_t offn) {
    if (!pre || jn >= a.pre_nparts) return;
    pf_tot = __ldg(pcnt + jn);
    pf_e0 = offn + pl < a.pre_capg ? __ldg(pbase + offn + pl) : 0u;
    pf_e1 = offn + pl + pS < a.pre_capg ? __ldg(pbase + offn + pl + pS) : 0u;
  };
  // the pre-sampler's buckets are complete from here on (a no-op unless this
  // launch is its programmatic dependent; the initial frame above overlaps it)
  asm volatile("griddepcontrol.wait;" ::: "memory");
  prefetch(0, 0);

  // ---- the program, window by window
  const uint32_t* wp = nullptr;
  bool need_window = true;
  bool done = false;
  while (!done) {
    if (need_window) {
      const bool ok = mbar_wait(&bars[kwin & 1], (uint32_t)((kwin >> 1) & 1));
      if (__syncthreads_or(!ok)) {  // every thread takes the same branch
        if (tid == 0) atomicExch(a.err, QCB_ETIMEOUT);
        return false;
      }
      wp = (kwin & 1) ? win1 : win0;
      need_window = false;
    }
    __syncthreads();  // the tile init / the previous record is complete
    const uint4 h = *(const uint4*)wp;
    const uint32_t kind = h.x >> 24, cnt = h.x & 0xFFFFFFu;
    const uint32_t* e = wp + 4;
    switch (kind) {
      case SEG_END:
        done = true;
        break;
      case SEG_WIN:
        break;
      case SEG_CNOT: {
        wp = e + ((cnt * 2 + 3) & ~3u);
        if (!act) break;
        const uint2* en = (const uint2*)e;
        uint32_t j = rr;
        for (; j + R < cnt; j += 2 * R) {
          const uint2 o = en[j], u = en[j + R];
          uint2 *pxc = F.at2(o.x & 0xFFFFu, cw, cg), *pzc = F.at2(o.x >> 16, cw, cg);
          uint2 *pxt = F.at2(o.y & 0xFFFFu, cw, cg), *pzt = F.at2(o.y >> 16, cw, cg);
          uint2 *qxc = F.at2(u.x & 0xFFFFu, cw, cg), *qzc = F.at2(u.x >> 16, cw, cg);
          uint2 *qxt = F.at2(u.y & 0xFFFFu, cw, cg), *qzt = F.at2(u.y >> 16, cw, cg);
          const uint2 xc = *pxc, zc = *pzc, xt = *pxt, zt = *pzt;
          const uint2 yxc = *qxc, yzc = *qzc, yxt = *qxt, yzt = *qzt;
          *pxt = xor2(xt, xc); *pzc = xor2(zc, zt);
          *qxt = xor2(yxt, yxc); *qzc = xor2(yzc, yzt);
        }
        for (; j < cnt; j += R) {
          const uint2 o = en[j];
          uint2 *pxc = F.at2(o.x & 0xFFFFu, cw, cg), *pzc = F.at2(o.x >> 16, cw, cg);
          uint2 *pxt = F.at2(o.y & 0xFFFFu, cw, cg), *pzt = F.at2(o.y >> 16, cw, cg);
          const uint2 xc = *pxc, zc = *pzc, xt = *pxt, zt = *pzt;
          *pxt = xor2(xt, xc); *pzc = xor2(zc, zt);
        }
        break;
      }
      case SEG_CZ: {
        wp = e + ((cnt * 2 + 3) & ~3u);
        if (!act) break;
        const uint2* en = (const uint2*)e;
        for (uint32_t j = rr; j < cnt; j += R) {
          const uint2 o = en[j];
          uint2 *pxa = F.at2(o.x & 0xFFFFu, cw, cg), *pza = F.at2(o.x >> 16, cw, cg);
          uint2 *pxb = F.at2(o.y & 0xFFFFu, cw, cg), *pzb = F.at2(o.y >> 16, cw, cg);
          const uint2 xa = *pxa, za = *pza, xb = *pxb, zb = *pzb;
          *pza = xor2(za, xb); *pzb = xor2(zb, xa);
        }
        break;
      }
      case SEG_S:
      case SEG_G1: {
        wp = e + ((cnt * 2 + 3) & ~3u);
        if (!act) break;
        const uint2* en = (const uint2*)e;
        for (uint32_t j = rr; j < cnt; j += R) {
          const uint2 o = en[j];
          uint2 *px = F.at2(o.x & 0xFFFFu, cw, cg), *pz = F.at2(o.x >> 16, cw, cg);
          uint2 x = *px, z = *pz;
          if (kind == SEG_S) {
            z = xor2(z, x);
          } else {
            gate1_xz(o.y, x.x, z.x);
            gate1_xz(o.y, x.y, z.y);
          }
          *px = x; *pz = z;
        }
        break;
      }
      case SEG_G2: {
        wp = e + cnt * 4;
        if (!act) break;
        const uint4* en = (const uint4*)e;
        for (uint32_t j = rr; j < cnt; j += R) {
          const uint4 o = en[j];
          uint2 *pxa = F.at2(o.x & 0xFFFFu, cw, cg), *pza = F.at2(o.x >> 16, cw, cg);
          uint2 *pxb = F.at2(o.y & 0xFFFFu, cw, cg), *pzb = F.at2(o.y >> 16, cw, cg);
          uint2 xa = *pxa, za = *pza, xb = *pxb, zb = *pzb;
          gate2_xz(o.z, xa.x, za.x, xb.x, zb.x);
          gate2_xz(o.z, xa.y, za.y, xb.y, zb.y);
          *pxa = xa; *pza = za; *pxb = xb; *pzb = zb;
        }
        break;
      }
      case SEG_MZ: {
        wp = e + ((cnt * 2 + 3) & ~3u);
        if (!act) break;
        const uint2* en = (const uint2*)e;
        for (uint32_t j = rr; j < cnt; j += R) {
          const uint2 o = en[j];
          *(uint2*)(a.rec + (uint64_t)o.y * rpitch + cg) = *F.at2(o.x, cw, cg);
        }
        break;
      }
      case SEG_MRZ: {
        wp = e + cnt * 16;
        if (!act) break;
        const uint4* en = (const uint4*)e;
        for (uint32_t g = rr; g < cnt; g += R) {
          uint4 ent[4];
#pragma unroll
          for (int i = 0; i < 4; i++) ent[i] = en[4 * g + i];
          uint32_t o[4] = {0, 0, 0, 0}, u[4] = {0, 0, 0, 0};
          if (PHILOX) {
            uint32_t blk = 0;
#pragma unroll
            for (int i = 0; i < 4; i++)
              if (ent[i].z != MRZ_PAD) blk = ent[i].z >> 2;
            philox4x32_10(blk, clo, chi, TAG_RESET, k0, k1, o);
            philox4x32_10(blk, clo1, chi1, TAG_RESET, k0, k1, u);
          }
#pragma unroll
          for (int i = 0; i < 4; i++) {
            if (ent[i].z == MRZ_PAD) continue;
            uint2* px = F.at2(ent[i].x & 0xFFFFu, cw, cg);
            uint2* pz = F.at2(ent[i].x >> 16, cw, cg);
            const uint2 x = *px, z = *pz;
            uint2 rb = make_uint2(o[i], u[i]);
            if (!PHILOX) {
              const uint32_t* rp = a.reset_planes + (uint64_t)ent[i].z * a.reset_pitch + cg;
              rb = a.reset_planes ? make_uint2(__ldg(rp), two ? __ldg(rp + 1) : 0u) : make_uint2(0u, 0u);
            }
            if (ent[i].y != BIT_NONE) *(uint2*)(a.rec + (uint64_t)ent[i].y * rpitch + cg) = x;
            *px = make_uint2(0u, 0u);
            *pz = xor2(z, rb);
          }
        }
        break;
      }
      case SEG_XOR: {
        wp = e + cnt * 32;
        if (!act) break;
        for (uint32_t j = rr; j < cnt; j += R) {
          const uint32_t* x = e + 32 * j;  // (store, n, b_0 .. b_{n-1})
          const uint32_t n = min(x[1], XOR_MAX_BITS);
          uint2 v = make_uint2(0u, 0u);
          for (uint32_t i = 0; i < n; i++) v = xor2(v, *(const uint2*)(a.rec + (uint64_t)x[2 + i] * rpitch + cg));
          *(uint2*)(a.rec + (uint64_t)x[0] * rpitch + cg) = v;
        }
        break;
      }
      case SEG_FLUSH: {
        wp = e + cnt * 4;
        const uint4* en = (const uint4*)e;
        if (PHILOX) {
          if (a.pmax > 0.0) {
            // (site, shot group) tasks over all threads of the CTA; a group
            // is 32 run columns and may straddle the tile's edges
            const uint64_t gc0 = a.col0 + c0;
            const uint64_t gc1 = a.col0 + min(c0 + T, a.ncols);
            const uint64_t G0 = gc0 / 32;
            const uint32_t ng = (uint32_t)((gc1 - 1) / 32 - G0 + 1);
            const uint32_t ntask = cnt * ng;
            // t / ng as a multiply-high for ng >= 2: ng <= 10 and t < 2^13 (a
            // record part fits one window), far inside t * (mg * ng - 2^32) < 2^32
            const uint32_t mg = ng > 1 ? 0xFFFFFFFFu / ng + 1u : 0u;
            if (PRE && a.pre_buf) {
              // pre-sampled: bucket (group G0 + pgl, part j), the count and
              // first events loaded at the previous flush part
              const uint32_t j = h.z, off = h.w, cap = h.y >> 8;
              const uint32_t total = pf_tot, ev0 = pf_e0, ev1 = pf_e1;
              prefetch(j + 1, off + cap);
              if (pre && cap) {
                const uint32_t* bk = pbase + off;
                const int32_t lc0 = (int32_t)((int64_t)((pG0 + pgl) * 32) - (int64_t)gc0);
                if (total <= cap) {
                  for (uint32_t m = pl; m < total; m += pS) {
                    const uint32_t ev = m == pl ? ev0 : m == pl + pS ? ev1 : __ldg(bk + m);
                    apply_code<SMEM>(F, en[ev >> 16], (ev >> 10) & 15u, lc0, ev & (NOISE_GROUP - 1), c0, a.ncols);
                  }
                } else {  // the bucket overflowed: draw its sparse sites here
                  for (uint32_t i = pl; i < cnt; i += pS)
                    if (!a.classes[en[i].y >> 8].dense) sample_site_group<SMEM>(a, F, en[i], pG0 + pgl, lc0, c0);
                }
              }
              if (h.y & FLAG_DENSE_SITES) {  // dense sites are drawn in the walk
                for (uint32_t t = tid; t < ntask; t += blockDim.x) {
                  const uint32_t i = ng > 1 ? __umulhi(t, mg) : t, gt = t - i * ng;
                  if (!a.classes[en[i].y >> 8].dense) continue;
                  const int32_t lc0 = (int32_t)((int64_t)((G0 + gt) * 32) - (int64_t)gc0);
                  sample_site_group<SMEM>(a, F, en[i], G0 + gt, lc0, c0);
                }
              }
            } else {
              for (uint32_t t = tid; t < ntask; t += blockDim.x) {
                const uint32_t i = ng > 1 ? __umulhi(t, mg) : t, gl = t - i * ng;
                const int32_t lc0 = (int32_t)((int64_t)((G0 + gl) * 32) - (int64_t)gc0);
                sample_site_group<SMEM>(a, F, en[i], G0 + gl, lc0, c0);
              }
            }
          }
        } else if (rr == 0 && act) {
          // each column's events are sorted by trial (site*32 + lane)
          for (uint32_t hc = 0; hc < 2; hc++) {
            const uint64_t eb = ep[hc], ee = ep[hc + 1];
            if (eb == ee) continue;
            for (uint32_t i = 0; i < cnt; i++) {
              const uint4 st = en[i];
              const uint64_t lo_t = (uint64_t)st.x * 32u, lim = lo_t + 32u;
              uint64_t lo = eb, hi = ee;
              while (lo < hi) {
                const uint64_t mid = (lo + hi) >> 1;
                if ((__ldg(a.ev_data + mid) >> 8) < lo_t) lo = mid + 1;
                else hi = mid;
              }
              for (uint64_t k = lo; k < ee; k++) {
                const uint64_t d = __ldg(a.ev_data + k);
                const uint64_t t = d >> 8;
                if (t >= lim) break;
                const uint32_t code = (uint32_t)(d & 0xFF), bit = 1u << (t & 31);
                if (code & 1) *F.at32(st.z & 0xFFFFu, cw + hc, cg + hc) ^= bit;
                if (code & 2) *F.at32(st.z >> 16, cw + hc, cg + hc) ^= bit;
                if ((st.y & 0xFFu) == QCB_OP_DEPOL2) {
                  if (code & 4) *F.at32(st.w & 0xFFFFu, cw + hc, cg + hc) ^= bit;
                  if (code & 8) *F.at32(st.w >> 16, cw + hc, cg + hc) ^= bit;
                }
              }
            }
          }
        }
        break;
      }
      default:
        done = true;
        break;
    }
    if (kind == SEG_WIN || kind == SEG_END) {
      __syncthreads();  // every thread is done with this window
      if (tid == 0) issue(kwin + 2);
      kwin++;
      need_window = true;
      if (kind == SEG_END) break;
    }
  }

  // ---- write the frame back, undoing the x<->z relabels
  for (uint32_t s = rr; s < a.nslots; s += R) {
    if (!act) break;
    const uint32_t q = __ldg(a.slot_qubit + s), sw = __ldg(a.slot_swap + s);
    uint2* gx = (uint2*)(a.planes + (uint64_t)(2 * q) * pitch + cg);
    uint2* gz = (uint2*)(a.planes + (uint64_t)(2 * q + 1) * pitch + cg);
    if (SMEM) {
      *gx = *F.at2(2 * s + sw, cw, cg);
      *gz = *F.at2(2 * s + 1 - sw, cw, cg);
    } else if (sw) {
      const uint2 x = *gx, z = *gz;
      *gx = z;
      *gz = x;
    }
  }
  __syncthreads();
  return true;
}

// Threads of a plain walker CTA at most (its launch bound): 640 leaves 96
// registers a thread, where the pre-sampled flush and its loads one part
// ahead fit without spilling (768 left 80 and spilled: d=11 0.69 against
// 0.59 ms per step).
constexpr uint32_t WALKER_THREADS = 640;

// The plain launch: one program on one frame, CTA b walking tiles b, b + grid, ...
template <bool SMEM, bool PHILOX>
__global__ void __launch_bounds__(WALKER_THREADS, 1) walker_kernel(const WalkArgs a) {
  extern __shared__ __align__(128) uint32_t sm[];
  const uint32_t tid = threadIdx.x, T = a.tile;
  // layout: [frame tile | pmap] [window 0] [window 1] [2 mbarriers]
  const uint32_t tile_words = SMEM ? 2 * a.nslots * T : 2 * a.nslots;
  uint32_t* win0 = sm + ((tile_words + 31) & ~31u);
  uint32_t* win1 = win0 + a.win_words;
  uint64_t* bars = (uint64_t*)(win1 + a.win_words);
  if (!SMEM)
    for (uint32_t p = tid; p < 2 * a.nslots; p += blockDim.x) sm[p] = 2 * a.slot_qubit[p >> 1] + (p & 1);
  const uint64_t ntiles = (a.ncols + T - 1) / T;
  const uint64_t my_tiles = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const uint64_t total_win = my_tiles * a.nwin;  // windows this CTA walks
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // window k of the flattened (tile, window) sequence lives in buffer k & 1
  auto issue = [&](uint64_t k) {
    if (k >= total_win || (a.withhold && k == a.withhold)) return;
    const uint32_t w = (uint32_t)(k % a.nwin);
    stage_window((k & 1) ? win1 : win0, a.prog + (size_t)w * (a.win_words / 4), a.win_words * 4, &bars[k & 1]);
  };
  if (tid == 0) { issue(0); issue(1); }
  uint64_t kwin = 0;
  bool failed = false;
  for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    if (!walk_tile<SMEM, PHILOX, PHILOX>(a, sm, win0, win1, bars, kwin, issue, tile)) {
      failed = true;
      break;
    }
  }
  // no bulk copy may still be in flight when the CTA exits
  if (failed) {
    __syncthreads();
    if (tid == 0)
      for (uint64_t k = kwin; k < kwin + 2 && k < total_win; k++) mbar_wait(&bars[k & 1], (uint32_t)((k >> 1) & 1));
  }
}

// ---------------------------------------------------------------- batches
// Many (program, frame) jobs drained from one persistent launch: the items
// are (job, tile) pairs in a queue ordered longest first; each CTA (one per
// SM) takes the next item with an atomic on the queue head.  Thread 0 stages
// program windows two ahead across item boundaries: when it stages the last
// window of an item it takes the next item and records it in a ring that the
// walk reads when it reaches that item.  Every job is fresh (initZ! fused)
// and in Philox mode, so its results are those of its plain launch.
struct BatchItem {
  uint32_t job;
  uint32_t pad;
  uint64_t tile;
};

struct BatchArgs {
  const WalkArgs* jobs;
  const BatchItem* items;
  uint32_t nitems;
  uint32_t tile_words;  // the largest frame tile of the jobs (words)
  uint32_t* head;       // next queue item (zero before the launch)
  uint32_t win_words;   // the largest program window of the jobs (words): the staging buffers' size
  uint32_t pad_;
};

constexpr uint32_t ITEM_NONE = 0xFFFFFFFFu;
static_assert(sizeof(WalkArgs) % 8 == 0, "WalkArgs is copied in 8-byte words");

__global__ void __launch_bounds__(768, 1) batch_walker_kernel(const BatchArgs b) {
  extern __shared__ __align__(128) uint32_t sm[];
  __shared__ uint32_t itemq[8];
  __shared__ __align__(16) WalkArgs ja;
  const uint32_t tid = threadIdx.x;
  uint32_t* win0 = sm + ((b.tile_words + 31) & ~31u);
  uint32_t* win1 = win0 + b.win_words;
  uint64_t* bars = (uint64_t*)(win1 + b.win_words);
  // staging side (thread 0): the item being staged and its next window
  uint32_t icur = ITEM_NONE, iw = 0, iq = 0;
  uint64_t issued = 0;
  auto fetch = [&]() -> uint32_t {
    const uint32_t i = atomicAdd(b.head, 1u);
    return i < b.nitems ? i : ITEM_NONE;
  };
  auto issue = [&](uint64_t) {
    if (icur == ITEM_NONE) return;
    const WalkArgs& J = b.jobs[b.items[icur].job];
    stage_window((issued & 1) ? win1 : win0, J.prog + (size_t)iw * (J.win_words / 4), J.win_words * 4,
                 &bars[issued & 1]);
    issued++;
    if (++iw == J.nwin) {
      iw = 0;
      icur = fetch();
      iq++;
      itemq[iq & 7] = icur;
    }
  };
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    icur = fetch();
    itemq[0] = icur;
    issue(0);
    issue(1);
  }
  __syncthreads();
  uint64_t kwin = 0;
  bool failed = false;
  for (uint32_t wi = 0;; wi++) {
    const uint32_t it = itemq[wi & 7];  // staged at least one window earlier
    if (it == ITEM_NONE) break;
    const BatchItem bi = b.items[it];
    __syncthreads();  // everyone has read the ring and is done with the previous job
    for (uint32_t w = tid; w < sizeof(WalkArgs) / 8; w += blockDim.x)
      ((uint64_t*)&ja)[w] = ((const uint64_t*)(b.jobs + bi.job))[w];
    __syncthreads();
    if (!walk_tile<true, true, false>(ja, sm, win0, win1, bars, kwin, issue, bi.tile)) {
      failed = true;
      break;
    }
  }
  // no bulk copy may still be in flight when the CTA exits
  if (failed) {
    __syncthreads();
    if (tid == 0)
      for (uint64_t k = kwin; k < issued; k++) mbar_wait(&bars[k & 1], (uint32_t)((k >> 1) & 1));
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
// Outputs [o0, o0 + n) of the column-major frames x nbits Bool matrix
// (output o = bit (o / S), frame (o % S)) into out[0, n): four consecutive
// outputs per thread, one 32-bit store when all four are in range.
__global__ void record_to_bools_kernel(const uint32_t* rec, uint64_t pitch, uint64_t S, uint64_t o0,
                                       uint64_t n, uint8_t* out) {
  const uint64_t t = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * 4;
  if (t >= n) return;
  uint64_t b = (o0 + t) / S, fr = (o0 + t) - b * S;
  uint32_t v = 0;
  const uint32_t m = (uint32_t)(n - t < 4 ? n - t : 4);
  for (uint32_t k = 0; k < m; k++) {
    v |= ((__ldg(rec + b * pitch + (fr >> 5)) >> (fr & 31)) & 1u) << (8 * k);
    if (++fr == S) { fr = 0; b++; }
  }
  if (m == 4) *(uint32_t*)(out + t) = v;
  else for (uint32_t k = 0; k < m; k++) out[t + k] = (uint8_t)(v >> (8 * k));
}

// The inverse: record word (bit b, column c) from 32 Bools of the column-major
// frames x nbits matrix (bytes other than 0 count as true; padding shots 0).
__global__ void bools_to_record_kernel(const uint8_t* in, uint64_t S, uint32_t nbits, uint32_t* rec,
                                       uint64_t pitch, uint64_t ncols) {
  const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t b = blockIdx.y;
  if (c >= ncols) return;
  const uint8_t* src = in + (uint64_t)b * S + c * 32;
  uint32_t w = 0;
  for (uint32_t k = 0; k < 32 && c * 32 + k < S; k++) w |= (src[k] ? 1u : 0u) << k;
  rec[(uint64_t)b * pitch + c] = w;
}

}  // namespace qcb

using namespace qcb;

// Staging of qcb_frame_download_measurements on one device.
constexpr uint64_t MEAS_STAGE = 32ull << 20;
struct MeasStage {
  uint8_t* buf[2] = {nullptr, nullptr};
  cudaStream_t copy = nullptr;
  cudaEvent_t expanded[2] = {}, copied[2] = {};
};

static int check_frame(const qcb_frame* f) {
  if (!f) return fail(QCB_EARG, "null frame");
  return QCB_OK;
}

// After a synchronising call: report a device-side wait that gave up.
static int frame_device_status(const qcb_frame* f) {
  int32_t h = 0;
  if (cudaMemcpy(&h, f->err, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return QCB_OK;
  if (h) return fail(h, "a device-side wait of the frame walker expired; the frame contents are not valid");
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
  f->pre_own = true;
  size_t pbytes = (size_t)2 * (f->nq1 + 1) * f->pitch * 4;
  size_t rbytes = (size_t)std::max<uint32_t>(nbits, 1) * f->pitch * 4;
  cudaError_t e = cudaMalloc(&f->planes, pbytes);
  if (e == cudaSuccess) e = cudaMalloc(&f->record, rbytes);
  if (e == cudaSuccess) e = cudaMalloc(&f->err, 16);
  if (e == cudaSuccess) e = cudaMemset(f->err, 0, 16);
  if (e == cudaSuccess) e = cudaMemset(f->planes, 0, pbytes);
  if (e == cudaSuccess) e = cudaMemset(f->record, 0, rbytes);
  if (e != cudaSuccess) {
    cudaFree(f->planes); cudaFree(f->record); cudaFree(f->err);
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
  cudaFree(f->err);
  cudaFree(f->pre);
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
  QCB_CUDA(cudaMemsetAsync(f->err, 0, 4, S(stream)));  // the frame is reinitialised
  uint32_t nt = 256;
  initz_kernel<<<(unsigned)((f->ncols + nt - 1) / nt), nt, 0, S(stream)>>>(
      f->planes, f->pitch, f->ncols, f->nq1, seed, shot_offset / 32);
  QCB_LAUNCHED();
  return QCB_OK;
}

int qcb_frame_init_z_planes(qcb_frame* f, const uint32_t* z, void* stream) {
  if (int st = check_frame(f)) return st;
  if (!f->ncols) return QCB_OK;
  QCB_CUDA(cudaMemsetAsync(f->err, 0, 4, S(stream)));  // the frame is reinitialised
  // x planes to zero, z planes from the caller (strided 2D copy)
  QCB_CUDA(cudaMemset2DAsync(f->planes, 2 * f->pitch * 4, 0, f->ncols * 4, f->nq1, S(stream)));
  QCB_CUDA(cudaMemcpy2DAsync(f->planes + f->pitch, 2 * f->pitch * 4, z, f->ncols * 4,
                             f->ncols * 4, f->nq1, cudaMemcpyHostToDevice, S(stream)));
  QCB_CUDA(cudaStreamSynchronize(S(stream)));
  return QCB_OK;
}

int qcb_frame_clear(qcb_frame* f, void* stream) {
  if (int st = check_frame(f)) return st;
  QCB_CUDA(cudaMemsetAsync(f->err, 0, 4, S(stream)));
  QCB_CUDA(cudaMemsetAsync(f->planes, 0, (size_t)2 * (f->nq1 + 1) * f->pitch * 4, S(stream)));
  QCB_CUDA(cudaMemsetAsync(f->record, 0, (size_t)std::max<uint32_t>(f->nbits, 1) * f->pitch * 4, S(stream)));
  return QCB_OK;
}

// copy(frame) (src/pauli_frames.jl:17): planes and record, device to device.
int qcb_frame_copy(qcb_frame* dst, const qcb_frame* src, void* stream) {
  if (int st = check_frame(dst)) return st;
  if (int st = check_frame(src)) return st;
  if (dst->frames != src->frames || dst->nq1 != src->nq1 || dst->nbits != src->nbits)
    return fail(QCB_EDIM, "qcb_frame_copy: frames of different shapes");
  QCB_CUDA(cudaMemcpyAsync(dst->planes, src->planes, (size_t)2 * (src->nq1 + 1) * src->pitch * 4,
                           cudaMemcpyDeviceToDevice, S(stream)));
  QCB_CUDA(cudaMemcpyAsync(dst->record, src->record, (size_t)std::max<uint32_t>(src->nbits, 1) * src->pitch * 4,
                           cudaMemcpyDeviceToDevice, S(stream)));
  return QCB_OK;
}

}  // extern "C"

namespace qcb {

// Launch configuration for the walker (shared-memory tile when the touched
// qubits of a tile of >= 64 columns fit, else HBM planes).
struct WalkConfig {
  bool smem;
  uint32_t T;     // tile columns
  uint32_t nth;   // threads per CTA
  uint32_t grid;
  size_t smem_bytes;
};

static uint32_t g_tile_override = 0;
static uint32_t g_stage_withhold = 0;     // test knob, see WalkArgs::withhold
static uint32_t g_presample = 0;          // 0: automatic, 1: never, 2: every bucket overflows (test)
// Largest pre-sampler scratch (event buckets + counts) per frame; a run that
// needs more draws its noise in the walk.
constexpr uint64_t PRESAMPLE_MAX_BYTES = 512ull << 20;
static uint32_t g_threads_override = 0;  // threads per CTA (0: WALKER_THREADS)
static uint32_t g_walker_pdl = 1;        // the walker as a programmatic dependent of the pre-sampler
static uint32_t g_walker_narrow = 1;     // 8..14-column shared-memory tiles for tall programs (0: HBM planes)

// Tile width (even: threads own column pairs) for ncols columns with tiles of
// at most tmax columns: the fewest waves of one CTA per SM, then the narrowest
// tile that still needs no more waves, so that the last wave is as full as
// the others.  (The walker on HBM planes.)
static uint32_t balanced_tile(uint64_t ncols, uint32_t tmax) {
  tmax &= ~1u;
  const uint64_t nsm = (uint64_t)std::max(device_sm_count(), 1);
  const uint64_t waves = std::max<uint64_t>(1, (ncols + nsm * tmax - 1) / (nsm * tmax));
  const uint64_t t = ((ncols + nsm * waves - 1) / (nsm * waves) + 1) & ~1ull;
  return (uint32_t)std::min<uint64_t>(tmax, std::max<uint64_t>(t, 16));
}

// Tile width of the shared-memory walker: the even width in [16, tmax] with
// the least waves x (25 + k T), the cost model of a CTA that these launches
// fit (a fixed part worth about 25 columns, the program's walk, and a part
// per column), with k = 0.75 for power-of-two widths, whose warps' column
// pairs cover whole rows of the tile and so meet no shared-memory bank
// conflicts, 1.1 for 18 columns (nine pairs a row) and 1 otherwise; ties go
// to the wider tile.  Measured on surface-code memory circuits (2^21 shots,
// ms): d = 17: 32 columns 4.53, 42 (fewest waves) 5.29; d = 19: 32 5.98, 34
// 8.02; d = 21: 28 14.36, 16 16.75; d = 23: 22 20.21, 16 20.73; d = 25: 16
// 24.77, 18 28.69; d = 15 (2^22 shots): 56 7.96, 32 9.90; all of them the
// model's choice.
static uint32_t smem_tile(uint64_t ncols, uint32_t tmax, uint32_t tmin = 16) {
  tmax &= ~1u;
  const uint64_t nsm = (uint64_t)std::max(device_sm_count(), 1);
  uint32_t best = tmin;
  uint64_t best_cost = UINT64_MAX;
  for (uint32_t t = tmin; t <= tmax; t += 2) {
    const uint64_t waves = ((ncols + t - 1) / t + nsm - 1) / nsm;
    const uint64_t k = (t & (t - 1)) == 0 ? 75 : t == 18 ? 110 : 100;
    const uint64_t cost = waves * (2500 + k * t);
    if (cost <= best_cost) { best = t; best_cost = cost; }
  }
  return best;
}

// The plain walker's autotuner table (qcb_tune_walker): the fastest tile
// width and threads per CTA measured for a program size class (touched
// qubits) at a frame width (columns); used by runs of exactly that width.
struct WalkerTune {
  uint32_t T, threads;
};
static std::map<std::pair<uint32_t, uint64_t>, WalkerTune> g_tuned_walker;
static std::mutex g_tuned_walker_mu;

// Shared-memory tile when 2 planes x 16 columns of every touched qubit fit,
// else the same walker on the HBM planes.
static WalkConfig walk_config(const qcb_program* p, const qcb_frame* f) {
  WalkConfig wc{};
  const size_t per_col = (size_t)2 * std::max<uint32_t>(p->nslots, 1) * 4;
  const size_t stage = (size_t)2 * p->win_words * 4 + 16 + 128;  // windows, mbarriers, alignment
  const size_t maxsm = (size_t)device_max_smem_optin();
  const size_t budget = maxsm > stage ? maxsm - stage : 0;
  uint32_t T = 0;
  uint32_t tuned_threads = 0;
  if (!g_tile_override && !g_threads_override) {
    std::lock_guard<std::mutex> lk(g_tuned_walker_mu);
    auto it = g_tuned_walker.find({p->nslots, f->ncols});
    if (it != g_tuned_walker.end() && per_col * it->second.T <= budget) {
      T = it->second.T;
      tuned_threads = it->second.threads;
    }
  }
  if (T) {
  } else if (g_tile_override && per_col * g_tile_override <= budget) {
    T = g_tile_override;
  } else if (budget / per_col >= 16) {
    T = smem_tile(f->ncols, (uint32_t)std::min<size_t>(256, budget / per_col));
  } else if (g_walker_narrow && budget / per_col >= 8) {
    // tall programs (d >= 29 surface codes): 8..14-column tiles keep the
    // frame in shared memory instead of walking the HBM planes
    T = smem_tile(f->ncols, (uint32_t)(budget / per_col), 8);
  }
  const uint32_t threads = g_threads_override ? g_threads_override : tuned_threads ? tuned_threads : WALKER_THREADS;
  if (T) {
    wc.smem = true;
    wc.T = T;
    wc.nth = (threads / (T / 2)) * (T / 2);  // column pairs; the kernel's launch bound is WALKER_THREADS
    wc.smem_bytes = per_col * T + stage;
  } else {
    wc.smem = false;
    wc.T = balanced_tile(f->ncols, 128);
    wc.nth = (threads / (wc.T / 2)) * (wc.T / 2);
    wc.smem_bytes = (size_t)2 * p->nslots * 4 + stage;
  }
  const uint64_t tiles = (f->ncols + wc.T - 1) / wc.T;
  wc.grid = (uint32_t)std::min<uint64_t>(tiles ? tiles : 1, 1u << 30);
  return wc;
}

// Scratch bytes the pre-sampler needs for ncols columns of program p (0:
// the program has no pre-sampled noise).
static uint64_t presample_need(const qcb_program* p, uint64_t ncols) {
  if (g_presample == 1 || p->pre_ent.empty() || p->pmax <= 0.0) return 0;
  const uint64_t ngroups = (ncols + 31) / 32;
  return (ngroups * p->pre_capoff.back() + ngroups * p->pre_nparts) * 4;
}

// Scratch bytes the pre-sampler needs for the frame (0: not used): at most
// PRESAMPLE_MAX_BYTES, unless the frame was handed a scratch that large.
static uint64_t presample_bytes(const qcb_frame* f, const qcb_program* p) {
  const uint64_t need = presample_need(p, f->ncols);
  if (need <= PRESAMPLE_MAX_BYTES) return need;
  return (f->pre && !f->pre_own && f->pre_bytes >= need) ? need : 0;
}

// Grow the frame's pre-sampler scratch (frames made by qcb_frame_create only;
// the first run of a frame allocates, later runs reuse it).
static int ensure_presample_scratch(qcb_frame* f, const qcb_program* p) {
  const uint64_t need = presample_bytes(f, p);
  if (!need || f->pre_bytes >= need || !f->pre_own) return QCB_OK;
  if (f->pre) QCB_CUDA(cudaFree(f->pre));
  f->pre = nullptr;
  f->pre_bytes = 0;
  QCB_CUDA(cudaMalloc(&f->pre, need));
  f->pre_bytes = need;
  return QCB_OK;
}

// Pre-sample the run's sparse noise into the frame's scratch (counts zeroed,
// then one presample_kernel launch) and point the walk at it; nothing when
// the scratch is absent or too small (the walk then draws the noise).
static int launch_presample(qcb_frame* f, const qcb_program* p, WalkArgs& a, cudaStream_t st) {
  const uint64_t need = presample_bytes(f, p);
  if (!need) return QCB_OK;
  if (int s = ensure_presample_scratch(f, p)) return s;
  if (f->pre_bytes < need) return QCB_OK;
  const uint64_t ngroups = (f->ncols + 31) / 32;
  const uint64_t cnt_words = ngroups * p->pre_nparts;
  PresampleArgs q{};
  q.ent = p->d_pre_ent;
  q.nent = (uint32_t)p->pre_ent.size();
  q.nparts = p->pre_nparts;
  q.g0 = a.col0 / 32;
  q.ngroups = ngroups;
  q.classes = p->d_classes;
  q.cdf = p->d_cdf;
  q.seed = a.seed;
  q.cnt = f->pre;
  q.buf = f->pre + cnt_words;
  q.capoff = p->d_pre_capoff;
  q.capg = p->pre_capoff.back();
  q.force_overflow = g_presample == 2 ? 1u : 0u;
  QCB_CUDA(cudaMemsetAsync(q.cnt, 0, cnt_words * 4, st));
  // each thread walks groups g, g + grid.y, ...: about 8 CTAs per SM in all
  const uint32_t gx = (q.nent + 255) / 256;
  const uint64_t gy = std::max<uint64_t>(1, ((uint64_t)device_sm_count() * 8 + gx - 1) / gx);
  const dim3 grid(gx, (uint32_t)std::min<uint64_t>(std::min<uint64_t>(ngroups, gy), 65535));
  presample_kernel<<<grid, 256, 0, st>>>(q);
  QCB_LAUNCHED();
  a.pre_buf = q.buf;
  a.pre_cnt = q.cnt;
  a.pre_capoff = p->d_pre_capoff;
  a.pre_nparts = p->pre_nparts;
  a.pre_capg = q.capg;
  return QCB_OK;
}

static void fill_common(WalkArgs& a, qcb_frame* f, const qcb_program* p);
int launch_walker(qcb_frame* f, const qcb_program* p, WalkArgs& a, bool philox, bool fresh, cudaStream_t st);

// Largest scratch of a chunked run (two chunks' event buckets).
constexpr uint64_t CHUNKED_PRESAMPLE_MAX = 4ull << 30;

// Columns per chunk of a Philox run whose pre-sampler scratch would pass
// PRESAMPLE_MAX_BYTES: whole walker waves (a whole number of 1024-shot
// groups), as many as fit twice over in PRESAMPLE_MAX_BYTES, at least one
// (strong noise on tall circuits: d = 21, p = 7.7e-3 needs about 0.5 GB a
// wave); 0 when two waves' scratch passes CHUNKED_PRESAMPLE_MAX (the run then
// draws its noise in the walk).
static uint64_t presample_chunk_cols(const qcb_program* p, const qcb_frame* f) {
  const uint64_t nsm = (uint64_t)std::max(device_sm_count(), 1);
  uint64_t unit = nsm * std::max<uint32_t>(walk_config(p, f).T, 1);
  while (unit % 32) unit *= 2;
  const uint64_t per = presample_need(p, unit);
  if (!per || 2 * per > CHUNKED_PRESAMPLE_MAX) return 0;
  const uint64_t budget = std::max<uint64_t>(PRESAMPLE_MAX_BYTES, 2 * per);
  uint64_t k = budget / (2 * per);
  while (k > 1 && 2 * presample_need(p, k * unit) > budget) k--;
  return k * unit;
}

// A side stream per device for the chunked runs below.
static cudaStream_t side_stream() {
  static std::mutex mu;
  static cudaStream_t streams[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  if (dev >= 0 && dev < 64 && !streams[dev]) cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking);
  return (dev >= 0 && dev < 64) ? streams[dev] : nullptr;
}

// A Philox run whose pre-sampler scratch would pass PRESAMPLE_MAX_BYTES, as
// column chunks of cw columns whose noise is pre-sampled (the frame keeps
// two scratches, one per chunk in flight): chunk k on the caller's stream
// (k even) or the side stream (k odd), forked from and joined back to the
// caller's stream, so that a chunk's last wave overlaps the next chunk.
// Columns are independent in Philox mode and every chunk counts with its
// global columns, so the frame and record equal those of one launch.
static int launch_walker_chunked(qcb_frame* f, const qcb_program* p, const WalkArgs& a0, bool fresh,
                                 cudaStream_t st, uint64_t cw) {
  const uint64_t half = (presample_need(p, cw) + 15) & ~15ull;
  if (f->pre_bytes < 2 * half) {
    if (f->pre) QCB_CUDA(cudaFree(f->pre));
    f->pre = nullptr;
    f->pre_bytes = 0;
    QCB_CUDA(cudaMalloc(&f->pre, 2 * half));
    f->pre_bytes = 2 * half;
  }
  cudaStream_t side = side_stream();
  if (!side) return fail(QCB_ECUDA, "no side stream for a chunked run");
  cudaEvent_t fork = nullptr, join = nullptr;
  QCB_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  QCB_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
  int status = QCB_OK;
  if (cudaEventRecord(fork, st) != cudaSuccess || cudaStreamWaitEvent(side, fork, 0) != cudaSuccess)
    status = fail(QCB_ECUDA, "chunked run: fork");
  for (uint64_t c0 = 0, k = 0; status == QCB_OK && c0 < f->ncols; c0 += cw, k++) {
    const uint64_t nc = std::min(cw, f->ncols - c0);
    qcb_frame view = *f;  // columns [c0, c0 + nc) of every plane and record row
    view.planes = f->planes + c0;
    view.record = f->record ? f->record + c0 : nullptr;
    view.ncols = nc;
    view.frames = nc * 32;
    view.pre = f->pre + (k & 1) * (half / 4);
    view.pre_bytes = half;
    view.pre_own = false;
    WalkArgs a;
    fill_common(a, &view, p);
    a.seed = a0.seed;
    a.col0 = a0.col0 + c0;
    status = launch_walker(&view, p, a, true, fresh, (k & 1) ? side : st);
  }
  if (cudaEventRecord(join, side) != cudaSuccess || cudaStreamWaitEvent(st, join, 0) != cudaSuccess)
    if (status == QCB_OK) status = fail(QCB_ECUDA, "chunked run: join");
  cudaEventDestroy(fork);
  cudaEventDestroy(join);
  return status;
}

int launch_walker(qcb_frame* f, const qcb_program* p, WalkArgs& a, bool philox, bool fresh,
                  cudaStream_t st) {
  if (philox && f->pre_own && f->ncols && presample_need(p, f->ncols) > PRESAMPLE_MAX_BYTES) {
    const uint64_t cw = presample_chunk_cols(p, f);
    if (cw && cw < f->ncols) return launch_walker_chunked(f, p, a, fresh, st, cw);
  }
  WalkConfig wc = walk_config(p, f);
  if (philox && f->ncols)
    if (int s = launch_presample(f, p, a, st)) return s;
  a.fresh = fresh ? 1 : 0;
  a.tile = wc.T;
  if (!f->ncols) return QCB_OK;
  void (*kern)(const WalkArgs);
  if (wc.smem) kern = philox ? walker_kernel<true, true> : walker_kernel<true, false>;
  else kern = philox ? walker_kernel<false, true> : walker_kernel<false, false>;
  if (wc.smem_bytes > 48 * 1024) {
    QCB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, device_max_smem_optin()));
    // all of the unified L1 / shared memory as shared memory, so that two
    // narrow tiles can share an SM when their frames fit side by side
    QCB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  (int)cudaSharedmemCarveoutMaxShared));
  }
  // after the pre-sampler, as its programmatic dependent
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(wc.grid);
  cfg.blockDim = dim3(wc.nth);
  cfg.dynamicSmemBytes = wc.smem_bytes;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = (a.pre_buf && g_walker_pdl) ? 1 : 0;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  QCB_CUDA(cudaLaunchKernelEx(&cfg, kern, (const WalkArgs)a));
  QCB_LAUNCHED();
  return QCB_OK;
}

static void fill_common(WalkArgs& a, qcb_frame* f, const qcb_program* p) {
  std::memset(&a, 0, sizeof(a));
  a.prog = (const uint4*)p->d_stream_slot;
  a.planes = f->planes;
  a.rec = f->record;
  a.pitch = f->pitch;
  a.rec_pitch = f->pitch;
  a.ncols = f->ncols;
  a.slot_qubit = p->d_slot_qubit;
  a.slot_swap = p->d_slot_swap;
  a.nslots = p->nslots;
  a.nq1 = f->nq1;
  a.qubit_slot = p->d_qubit_slot;
  a.qubit_slot_len = p->qubit_slot_len;
  a.prog = (const uint4*)p->d_stream_slot;
  a.win_words = p->win_words;
  a.nwin = (uint32_t)(p->stream_slot.size() / p->win_words);
  a.classes = p->d_classes;
  a.cdf = p->d_cdf;
  a.pmax = p->pmax;
  a.err = f->err;
  a.withhold = g_stage_withhold;
}

static int check_run(const qcb_frame* f, const qcb_program* p, const qcb_noise_source* n) {
  if (!f || !p || !n) return fail(QCB_EARG, "null argument");
  if (p->nq > f->nq1)
    return fail(QCB_EBOUNDS, "program uses qubit " + std::to_string(p->nq) + " but the frame has " +
                                 std::to_string(f->nq1) + " (qubits + hidden ancilla)");
  if (p->info.nbits > f->nbits)
    return fail(QCB_EBOUNDS, "program records bit " + std::to_string(p->info.nbits) +
                                 " but the frame has " + std::to_string(f->nbits));
  if (n->mode != QCB_NOISE_PHILOX && n->mode != QCB_NOISE_MASK) return fail(QCB_EARG, "bad noise mode");
  if (n->shot_offset % (n->mode == QCB_NOISE_PHILOX ? NOISE_GROUP : 32))
    return fail(QCB_EARG, "shot_offset must be a multiple of 1024 (Philox mode) or 32 (mask mode)");
  return QCB_OK;
}

int run_program(qcb_frame* f, const qcb_program* p, const qcb_noise_source* n, bool fresh,
                cudaStream_t st) {
  if (int s = check_run(f, p, n)) return s;
  WalkArgs a;
  fill_common(a, f, p);
  a.seed = n->seed;
  a.col0 = n->shot_offset / 32;
  // a fresh run rewrites the whole frame: an earlier expired wait no longer applies
  if (fresh) QCB_CUDA(cudaMemsetAsync(f->err, 0, 4, st));
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
  const uint64_t bytes = (uint64_t)f->frames * f->nbits;
  if (!bytes) return QCB_OK;
  // Expanded on the device in chunks of at most MEAS_STAGE bytes into two
  // staging buffers of the current device (allocated at its first call, kept
  // for the process), each chunk copied out on a second stream while the next
  // one expands; calls are serialised by a lock.
  static std::mutex mu;
  static std::map<int, MeasStage> stages;
  std::lock_guard<std::mutex> lock(mu);
  int dev = 0;
  QCB_CUDA(cudaGetDevice(&dev));
  MeasStage& g = stages[dev];
  if (!g.buf[0]) {
    QCB_CUDA(cudaMalloc(&g.buf[0], 2 * MEAS_STAGE));
    g.buf[1] = g.buf[0] + MEAS_STAGE;
    QCB_CUDA(cudaStreamCreateWithFlags(&g.copy, cudaStreamNonBlocking));
    for (int k = 0; k < 2; k++) {
      QCB_CUDA(cudaEventCreateWithFlags(&g.expanded[k], cudaEventDisableTiming));
      QCB_CUDA(cudaEventCreateWithFlags(&g.copied[k], cudaEventDisableTiming));
    }
  }
  cudaStream_t st = S(stream);
  uint64_t k = 0;
  for (uint64_t o0 = 0; o0 < bytes; o0 += MEAS_STAGE, k++) {
    const uint64_t n = std::min<uint64_t>(MEAS_STAGE, bytes - o0);
    const int b = (int)(k & 1);
    if (k >= 2) QCB_CUDA(cudaStreamWaitEvent(st, g.copied[b], 0));  // buffer b is free again
    const uint64_t threads = (n + 3) / 4;
    record_to_bools_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(f->record, f->pitch, f->frames, o0, n,
                                                                             g.buf[b]);
    QCB_LAUNCHED();
    QCB_CUDA(cudaEventRecord(g.expanded[b], st));
    QCB_CUDA(cudaStreamWaitEvent(g.copy, g.expanded[b], 0));
    QCB_CUDA(cudaMemcpyAsync(bools + o0, g.buf[b], n, cudaMemcpyDeviceToHost, g.copy));
    QCB_CUDA(cudaEventRecord(g.copied[b], g.copy));
  }
  QCB_CUDA(cudaStreamSynchronize(g.copy));
  QCB_CUDA(cudaStreamSynchronize(st));
  return frame_device_status(f);
}

int qcb_frame_upload_measurements(qcb_frame* f, const uint8_t* bools, void* stream) {
  if (int st = check_frame(f)) return st;
  const size_t bytes = (size_t)f->frames * f->nbits;
  if (!bytes) return QCB_OK;
  if (!bools) return fail(QCB_EARG, "null measurements");
  uint8_t* d = nullptr;
  QCB_CUDA(cudaMallocAsync(&d, bytes, S(stream)));
  QCB_CUDA(cudaMemcpyAsync(d, bools, bytes, cudaMemcpyHostToDevice, S(stream)));
  dim3 grid((unsigned)((f->ncols + 255) / 256), f->nbits);
  bools_to_record_kernel<<<grid, 256, 0, S(stream)>>>(d, f->frames, f->nbits, f->record, f->pitch, f->ncols);
  QCB_LAUNCHED();
  QCB_CUDA(cudaFreeAsync(d, S(stream)));
  QCB_CUDA(cudaStreamSynchronize(S(stream)));  // the caller's buffer may go after the call
  return QCB_OK;
}

int qcb_frame_download_record_planes(const qcb_frame* f, uint32_t* planes, void* stream) {
  if (int st = check_frame(f)) return st;
  if (!f->nbits || !f->ncols) return QCB_OK;
  QCB_CUDA(cudaMemcpy2DAsync(planes, f->ncols * 4, f->record, f->pitch * 4, f->ncols * 4, f->nbits,
                             cudaMemcpyDeviceToHost, S(stream)));
  QCB_CUDA(cudaStreamSynchronize(S(stream)));
  return frame_device_status(f);
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

}  // extern "C"

namespace qcb {

// Page-locked copy of a compiled program's device image (records, noise
// classes, count tables) for the one-call host API, which copies it to the
// device on every call.
struct HostProgramImage {
  uint8_t* pinned = nullptr;
  size_t cap = 0, n_stream = 0, n_classes = 0, n_cdf = 0;
  int build(const Program& P) {
    n_stream = P.stream_slot.size() * sizeof(uint32_t);
    n_classes = P.classes.size() * sizeof(NoiseClass);
    n_cdf = P.cdf.size() * sizeof(uint32_t);
    const size_t need = n_stream + n_classes + n_cdf;
    if (need > cap) {
      if (pinned) cudaFreeHost(pinned);
      pinned = nullptr;
      cap = 0;
      QCB_CUDA(cudaMallocHost((void**)&pinned, need ? need : 16));
      cap = need;
    }
    if (n_stream) std::memcpy(pinned, P.stream_slot.data(), n_stream);
    if (n_classes) std::memcpy(pinned + n_stream, P.classes.data(), n_classes);
    if (n_cdf) std::memcpy(pinned + n_stream + n_classes, P.cdf.data(), n_cdf);
    return QCB_OK;
  }
  int upload(const Program& P, cudaStream_t st) const {
    if (n_stream) QCB_CUDA(cudaMemcpyAsync(P.d_stream_slot, pinned, n_stream, cudaMemcpyHostToDevice, st));
    if (n_classes)
      QCB_CUDA(cudaMemcpyAsync(P.d_classes, pinned + n_stream, n_classes, cudaMemcpyHostToDevice, st));
    if (n_cdf) QCB_CUDA(cudaMemcpyAsync(P.d_cdf, pinned + n_stream + n_classes, n_cdf, cudaMemcpyHostToDevice, st));
    return QCB_OK;
  }
};

// Copy-out chunks of the one-call host API: the first is one wave of
// 16-column tiles, each next one twice as wide, the last takes the rest.
constexpr int HOST_MAX_CHUNKS = 8;

static std::vector<std::pair<uint64_t, uint64_t>> host_chunks(uint64_t ncols) {
  const uint64_t first = std::max<uint64_t>(32, (uint64_t)std::max(device_sm_count(), 1) * 16 / 32 * 32);
  std::vector<std::pair<uint64_t, uint64_t>> ch;
  if (ncols < 4 * first) {
    ch.push_back({0, ncols});
    return ch;
  }
  uint64_t c0 = 0, w = first;
  while (c0 < ncols) {
    const uint64_t nc = (int)ch.size() + 1 == HOST_MAX_CHUNKS ? ncols - c0 : std::min(w, ncols - c0);
    ch.push_back({c0, nc});
    c0 += nc;
    w *= 2;
  }
  return ch;
}

}  // namespace qcb

extern "C" {

// One-call pftrajectories(circuit; trajectories): program and frame are
// cached between calls (keyed by the op list and the frame shape).  With a
// host record the run is cut into shot chunks, launched in order on the
// caller's stream, and each chunk's record columns are copied to the host on
// a second stream as soon as that chunk is done: the PCIe copy, which bounds
// this call, starts after the first small chunk instead of after the whole
// run.  Chunk column offsets are multiples of 32 (1024-shot noise groups) and
// every chunk draws the Philox streams of its global columns, so the record
// equals that of one launch over all the shots.
int qcb_pftrajectories_host(const qcb_op* ops, size_t n_ops, uint64_t frames, uint64_t seed,
                            uint64_t shot_offset, uint32_t* record_planes, void* stream) {
  static std::mutex mu;
  static qcb_program* cprog = nullptr;
  static std::vector<qcb_op> cops;
  static qcb_frame* cframe = nullptr;
  static cudaStream_t copy_stream = nullptr;
  static cudaEvent_t chunk_done[HOST_MAX_CHUNKS + 1] = {};
  static HostProgramImage image;
  std::lock_guard<std::mutex> lock(mu);
  if (!cprog || cops.size() != n_ops || std::memcmp(cops.data(), ops, n_ops * sizeof(qcb_op)) != 0) {
    if (cprog) { qcb_program_destroy(cprog); cprog = nullptr; }
    if (int st = qcb_program_compile(ops, n_ops, &cprog)) return st;
    cops.assign(ops, ops + n_ops);
    if (int st = image.build(*cprog)) return st;
  }
  // The circuit is an input of every call: its compiled records, noise
  // classes and count tables go host -> device each call, from page-locked
  // memory, ahead of the walk on the same stream (the host-side compile is
  // what the op-list comparison saves).
  if (int st = image.upload(*cprog, S(stream))) return st;
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
  if (!record_planes) return run_program(cframe, cprog, &n, true, S(stream));
  if (int st = check_run(cframe, cprog, &n)) return st;
  if (!copy_stream) {
    QCB_CUDA(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
    for (cudaEvent_t& e : chunk_done) QCB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  const auto chunks = host_chunks(cframe->ncols);
  // the chunks share the frame's pre-sampler scratch, sized for the whole run
  if (int st = ensure_presample_scratch(cframe, cprog)) return st;
  for (size_t k = 0; k < chunks.size(); k++) {
    const uint64_t c0 = chunks[k].first, nc = chunks[k].second;
    qcb_frame view = *cframe;  // columns [c0, c0 + nc) of every plane
    view.pre_own = false;
    view.planes = cframe->planes + c0;
    view.record = cframe->record + c0;
    view.ncols = nc;
    view.frames = nc * 32;
    WalkArgs a;
    fill_common(a, &view, cprog);
    a.seed = seed;
    a.col0 = shot_offset / 32 + c0;
    if (int st = launch_walker(&view, cprog, a, true, true, S(stream))) return st;
    QCB_CUDA(cudaEventRecord(chunk_done[k], S(stream)));
    QCB_CUDA(cudaStreamWaitEvent(copy_stream, chunk_done[k], 0));
    QCB_CUDA(cudaMemcpy2DAsync(record_planes + c0, cframe->ncols * 4, cframe->record + c0, cframe->pitch * 4,
                               nc * 4, cframe->nbits, cudaMemcpyDeviceToHost, copy_stream));
  }
  QCB_CUDA(cudaEventRecord(chunk_done[HOST_MAX_CHUNKS], copy_stream));
  QCB_CUDA(cudaStreamWaitEvent(S(stream), chunk_done[HOST_MAX_CHUNKS], 0));
  QCB_CUDA(cudaStreamSynchronize(S(stream)));
  return frame_device_status(cframe);
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
void set_walker_tile(uint32_t t) { g_tile_override = t; }
void set_walker_pdl(uint32_t v) { g_walker_pdl = v; }
void set_walker_narrow(uint32_t v) { g_walker_narrow = v; }
void set_walker_threads(uint32_t t) { g_threads_override = t; }
void set_stage_withhold(uint32_t k) { g_stage_withhold = k; }
void set_presample(uint32_t v) { g_presample = v; }
int run_program_fresh(qcb_frame* f, const qcb_program* p, uint64_t seed, uint64_t shot_offset,
                      cudaStream_t st) {
  qcb_noise_source n{};
  n.mode = QCB_NOISE_PHILOX;
  n.seed = seed;
  n.shot_offset = shot_offset;
  return run_program(f, p, &n, true, st);
}
}  // namespace qcb

// ---------------------------------------------------------------- batches (host)
namespace qcb {

// The tuner's table: tile width per size class (touched qubits).
static std::map<uint32_t, uint32_t> g_tuned_tile;

// Widest tile (even, <= 256) whose frame fits one CTA's shared memory next to
// staging buffers of win_words words; 0 when not even 16 columns fit.
static uint32_t batch_tile_max(const qcb_program* p, uint32_t win_words) {
  const size_t per_col = (size_t)2 * std::max<uint32_t>(p->nslots, 1) * 4;
  const size_t stage = (size_t)2 * win_words * 4 + 16 + 128 + sizeof(WalkArgs) + 64;
  const size_t maxsm = (size_t)device_max_smem_optin();
  const size_t budget = maxsm > stage ? maxsm - stage : 0;
  uint32_t t = (uint32_t)std::min<size_t>(256, budget / per_col) & ~1u;
  return t >= 16 ? t : 0;
}

}  // namespace qcb

struct qcb_batch {
  std::vector<qcb_frame*> frames;
  qcb::WalkArgs* d_jobs = nullptr;
  qcb::BatchItem* d_items = nullptr;
  uint32_t* d_head = nullptr;
  uint32_t nitems = 0;
  uint32_t tile_words = 0;
  uint32_t win_words = 0;
  size_t smem_bytes = 0;
  uint32_t grid = 0;
};

extern "C" {

int qcb_batch_create(const qcb_batch_job* jobs, size_t n_jobs, qcb_batch** out) {
  using namespace qcb;
  if (!out || (n_jobs && !jobs)) return fail(QCB_EARG, "null argument");
  *out = nullptr;
  std::vector<WalkArgs> wa(n_jobs);
  struct Cost { double c; uint32_t job; uint64_t tile; };
  std::vector<Cost> items;
  uint32_t tile_words = 0;
  auto b = std::make_unique<qcb_batch>();
  // the staging buffers are shared by all jobs: the largest window of any job
  uint32_t win_words = PROG_WINDOW_WORDS;
  for (size_t j = 0; j < n_jobs; j++)
    if (jobs[j].program) win_words = std::max(win_words, jobs[j].program->win_words);
  for (size_t j = 0; j < n_jobs; j++) {
    const qcb_batch_job& J = jobs[j];
    qcb_noise_source n{};
    n.mode = QCB_NOISE_PHILOX;
    n.seed = J.seed;
    n.shot_offset = J.shot_offset;
    if (int s = check_run(J.frame, J.program, &n)) return s;
    const uint32_t tmax = batch_tile_max(J.program, win_words);
    if (!tmax) return fail(QCB_EUNSUPPORTED, "batch job " + std::to_string(j) + ": its frame tile does not fit shared memory");
    uint32_t T = J.tile;
    if (T && (T % 2 || T < 16 || T > tmax)) return fail(QCB_EARG, "batch job " + std::to_string(j) + ": bad tile width");
    if (!T) {
      auto it = g_tuned_tile.find(J.program->nslots);
      T = it != g_tuned_tile.end() ? std::min(it->second, tmax) : tmax;
    }
    const uint64_t ncols = J.frame->ncols;
    T = (uint32_t)std::min<uint64_t>(T, std::max<uint64_t>(16, (ncols + 1) & ~1ull));
    WalkArgs& a = wa[j];
    fill_common(a, J.frame, J.program);
    a.seed = J.seed;
    a.col0 = J.shot_offset / 32;
    a.fresh = 1;
    a.tile = T;
    tile_words = std::max(tile_words, 2 * J.program->nslots * T);
    b->frames.push_back(J.frame);
    // longest first: a tile walks every record once, its ops over T columns
    const double cost = (double)J.program->stream_slot.size() * (1.0 + T / 64.0);
    for (uint64_t t = 0; t * T < ncols; t++) items.push_back({cost, (uint32_t)j, t});
  }
  std::stable_sort(items.begin(), items.end(), [](const Cost& x, const Cost& y) { return x.c > y.c; });
  std::vector<BatchItem> it(items.size());
  for (size_t i = 0; i < items.size(); i++) it[i] = {items[i].job, 0u, items[i].tile};
  if (items.size() > 0xFFFFFFF0ull) return fail(QCB_EARG, "too many tiles in one batch");
  b->nitems = (uint32_t)items.size();
  b->tile_words = tile_words;
  b->win_words = win_words;
  b->smem_bytes = (size_t)((tile_words + 31) & ~31u) * 4 + (size_t)2 * win_words * 4 + 16;
  b->grid = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(b->nitems, 1), (uint64_t)device_sm_count());
  QCB_CUDA(cudaMalloc(&b->d_jobs, std::max<size_t>(wa.size(), 1) * sizeof(WalkArgs)));
  QCB_CUDA(cudaMalloc(&b->d_items, std::max<size_t>(it.size(), 1) * sizeof(BatchItem)));
  QCB_CUDA(cudaMalloc(&b->d_head, 4));
  if (!wa.empty()) QCB_CUDA(cudaMemcpy(b->d_jobs, wa.data(), wa.size() * sizeof(WalkArgs), cudaMemcpyHostToDevice));
  if (!it.empty()) QCB_CUDA(cudaMemcpy(b->d_items, it.data(), it.size() * sizeof(BatchItem), cudaMemcpyHostToDevice));
  QCB_CUDA(cudaFuncSetAttribute(batch_walker_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, device_max_smem_optin() - 1024));
  *out = b.release();
  return QCB_OK;
}

int qcb_batch_run(qcb_batch* b, void* stream) {
  using namespace qcb;
  if (!b) return fail(QCB_EARG, "null batch");
  if (!b->nitems) return QCB_OK;
  cudaStream_t st = S(stream);
  QCB_CUDA(cudaMemsetAsync(b->d_head, 0, 4, st));
  BatchArgs a{b->d_jobs, b->d_items, b->nitems, b->tile_words, b->d_head, b->win_words, 0u};
  batch_walker_kernel<<<b->grid, 768, b->smem_bytes, st>>>(a);
  QCB_LAUNCHED();
  return QCB_OK;
}

int qcb_batch_status(const qcb_batch* b) {
  if (!b) return fail(QCB_EARG, "null batch");
  for (qcb_frame* f : b->frames)
    if (int s = frame_device_status(f)) return s;
  return QCB_OK;
}

int qcb_batch_destroy(qcb_batch* b) {
  if (!b) return QCB_OK;
  cudaFree(b->d_jobs);
  cudaFree(b->d_items);
  cudaFree(b->d_head);
  delete b;
  return QCB_OK;
}

// The autotuner: time candidate tile widths for this program on a scratch
// frame of two full waves per candidate (fresh Philox runs, CUDA events) and
// keep the width with the most frame columns per second for the program's
// size class (its touched qubits); qcb_batch_create uses it.
int qcb_tune_walker(const qcb_program* p, uint64_t frames, uint32_t* tile_out, uint32_t* threads_out,
                    float* ms_out, void* stream) {
  using namespace qcb;
  if (!p) return fail(QCB_EARG, "null program");
  if (!frames) return fail(QCB_EARG, "qcb_tune_walker: frames must be > 0");
  const size_t per_col = (size_t)2 * std::max<uint32_t>(p->nslots, 1) * 4;
  const size_t stage = (size_t)2 * p->win_words * 4 + 16 + 128;
  const size_t maxsm = (size_t)device_max_smem_optin();
  const uint32_t tmax = maxsm > stage ? (uint32_t)std::min<size_t>(256, (maxsm - stage) / per_col) & ~1u : 0u;
  if (tmax < 8) return fail(QCB_EUNSUPPORTED, "the program's frame tile does not fit shared memory");
  const uint64_t ncols = (frames + 31) / 32;
  const uint32_t tmin = tmax >= 16 ? 16u : 8u;
  std::vector<uint32_t> tiles = {smem_tile(ncols, tmax, tmin)};
  for (uint32_t t : {8u, 16u, 32u, 64u, 128u, 256u})
    if (t >= tmin && t <= tmax && std::find(tiles.begin(), tiles.end(), t) == tiles.end()) tiles.push_back(t);
  const uint32_t threads[] = {448, 512, 576, 640};
  cudaStream_t st = S(stream);
  qcb_frame* f = nullptr;
  if (int s0 = qcb_frame_create(frames, p->nq > 0 ? p->nq - 1 : 0, p->info.nbits, &f)) return s0;
  cudaEvent_t e0, e1;
  QCB_CUDA(cudaEventCreate(&e0));
  QCB_CUDA(cudaEventCreate(&e1));
  const uint32_t saved_t = g_tile_override, saved_th = g_threads_override;
  uint32_t best_t = 0, best_th = 0;
  float best_ms = 0.f;
  int status = QCB_OK;
  for (uint32_t T : tiles) {
    for (uint32_t th : threads) {
      if (th / (T / 2) == 0) continue;
      g_tile_override = T;
      g_threads_override = th;
      float ms = 0.f;
      for (int rep = 0; rep < 4 && status == QCB_OK; rep++) {
        cudaEventRecord(e0, st);
        status = run_program_fresh(f, p, 0x5EEDull + rep, 0, st);
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) status = fail(QCB_ECUDA, "tuner timing");
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        if (rep > 0) ms = rep == 1 ? t : std::min(ms, t);  // rep 0 warms up
      }
      if (status != QCB_OK) break;
      if (!best_t || ms < best_ms) { best_t = T; best_th = th; best_ms = ms; }
    }
    if (status != QCB_OK) break;
  }
  g_tile_override = saved_t;
  g_threads_override = saved_th;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  qcb_frame_destroy(f);
  if (status != QCB_OK) return status;
  {
    std::lock_guard<std::mutex> lk(g_tuned_walker_mu);
    g_tuned_walker[{p->nslots, ncols}] = WalkerTune{best_t, best_th};
  }
  if (tile_out) *tile_out = best_t;
  if (threads_out) *threads_out = best_th;
  if (ms_out) *ms_out = best_ms;
  return QCB_OK;
}

int qcb_tune_walker_clear(void) {
  std::lock_guard<std::mutex> lk(qcb::g_tuned_walker_mu);
  qcb::g_tuned_walker.clear();
  return QCB_OK;
}

int qcb_tune_tile(const qcb_program* p, uint32_t* tile_out, float* us_per_column, void* stream) {
  using namespace qcb;
  if (!p) return fail(QCB_EARG, "null program");
  const uint32_t tmax = batch_tile_max(p, p->win_words);
  if (!tmax) return fail(QCB_EUNSUPPORTED, "the program's frame tile does not fit shared memory");
  cudaStream_t st = S(stream);
  const uint32_t cands[] = {16, 24, 32, 48, 64, 96, 128, 192, 256};
  const uint64_t nsm = (uint64_t)std::max(device_sm_count(), 1);
  uint32_t best = 0;
  float best_us = 0.f;
  cudaEvent_t e0, e1;
  QCB_CUDA(cudaEventCreate(&e0));
  QCB_CUDA(cudaEventCreate(&e1));
  const uint32_t saved = g_tile_override;
  int status = QCB_OK;
  for (uint32_t T : cands) {
    if (T > tmax) break;
    const uint64_t ncols = 2 * nsm * T;
    qcb_frame* f = nullptr;
    if ((status = qcb_frame_create(ncols * 32, p->nq > 0 ? p->nq - 1 : 0, p->info.nbits, &f))) break;
    g_tile_override = T;
    float ms = 0.f;
    for (int rep = 0; rep < 4 && status == QCB_OK; rep++) {
      cudaEventRecord(e0, st);
      status = run_program_fresh(f, p, 0x5EEDull + rep, 0, st);
      cudaEventRecord(e1, st);
      if (cudaEventSynchronize(e1) != cudaSuccess) status = fail(QCB_ECUDA, "tuner timing");
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      if (rep > 0) ms = rep == 1 ? t : std::min(ms, t);  // rep 0 warms up
    }
    qcb_frame_destroy(f);
    if (status != QCB_OK) break;
    const float us = ms * 1000.f / (float)ncols;
    if (!best || us < best_us) { best = T; best_us = us; }
  }
  g_tile_override = saved;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (status != QCB_OK) return status;
  g_tuned_tile[p->nslots] = best;
  if (tile_out) *tile_out = best;
  if (us_per_column) *us_per_column = best_us;
  return QCB_OK;
}

}  // extern "C"

// One shot chunk of a fresh Philox run for the serving loop: `f` holds the
// chunk's planes (its own record is not used), `ncols` columns of it are
// walked, and the chunk's record rows go to rec + b * rec_pitch (the chunk's
// columns of the request's full record).  Counters use the global column,
// so the chunks of a request give the record of one run over all its shots.
namespace qcb {
uint64_t chunk_presample_bytes(const qcb_program* p, uint64_t ncols) { return presample_need(p, ncols); }

void chunk_shape(const qcb_program* p, uint64_t ncols, uint32_t* tile, uint32_t* ctas) {
  qcb_frame view{};
  view.ncols = ncols;
  view.frames = ncols * 32;
  const WalkConfig wc = walk_config(p, &view);
  if (tile) *tile = wc.T;
  if (ctas) *ctas = wc.grid;
}

int run_chunk(qcb_frame* f, uint64_t ncols, const qcb_program* p, uint64_t seed, uint64_t shot_offset, uint32_t* rec,
              uint64_t rec_pitch, cudaStream_t st) {
  if (!f || !p || !rec) return fail(QCB_EARG, "null argument");
  if (p->nq > f->nq1) return fail(QCB_EBOUNDS, "program uses more qubits than the chunk frame has");
  if (ncols > f->ncols) return fail(QCB_EBOUNDS, "chunk wider than its frame");
  if (shot_offset % NOISE_GROUP) return fail(QCB_EARG, "chunk shot_offset must be a multiple of 1024");
  qcb_frame view = *f;
  view.ncols = ncols;
  view.frames = ncols * 32;
  WalkArgs a;
  fill_common(a, &view, p);
  a.rec = rec;
  a.rec_pitch = rec_pitch;
  a.seed = seed;
  a.col0 = shot_offset / 32;
  return launch_walker(&view, p, a, true, true, st);
}
}  // namespace qcb
