// program.cu -- circuit -> device program compiler.
//
// Replaces the per-op dispatch of pftrajectories(frame, circuit)
// (src/pauli_frames.jl:234-239) and compactify_circuit (src/sumtypes.jl:190-237).
//
//  * Ops are validated like the Julia constructors (NoZeroQubit, q1 == q2).
//  * sMX / sMRX are lowered to sHadamard + sMZ / sMRZ (src/pauli_frames.jl:74-83).
//  * Frames carry no phases (src/pauli_frames.jl:58-61), so sX/sY/sZ/sId1 do
//    nothing and are dropped, and the gates whose frame action is x <-> z
//    (sHadamard, sSQRTY, sInvSQRTY) cost nothing at run time: the compiler
//    keeps a per-qubit "swapped" flag and emits every later operand as the
//    physical plane that currently holds x or z.  The final flags are applied
//    when the frame is written back.
//  * The remaining ops are grouped into segments: runs of one kind on
//    pairwise-disjoint qubits.  Inside a segment all (op, shot column) pairs
//    are independent, so a thread block executes them in parallel and
//    synchronises once per segment.
//  * Noise ops do not break segments.  Their sites (with the planes current
//    at the noise op) are collected and applied at a FLUSH record placed before
//    the first later op that reads or writes one of their qubits; moving a
//    Pauli flip past ops on other qubits (or past a relabelling) is exact.
//  * Resets are grouped four at a time so that one Philox block serves four
//    resets of a shot column.
#include <cmath>
#include <cstring>
#include <algorithm>
#include <map>
#include <tuple>
#include <unordered_map>
#include <unordered_set>

#include "qcb_internal.h"

namespace qcb {

static bool is1q(uint32_t o) { return o >= QCB_OP_I && o <= QCB_OP_SQO; }
static bool is2q(uint32_t o) { return o >= QCB_OP_CNOT && o <= QCB_OP_LAST2Q; }
static bool isnoise(uint32_t o) { return o >= QCB_OP_PAULI_NOISE && o <= QCB_OP_DEPOL2; }
static bool ismeas(uint32_t o) { return o >= QCB_OP_MZ && o <= QCB_OP_MRX; }
// frame action x <-> z
static bool is_relabel(uint32_t o) { return o == QCB_OP_H || o == QCB_OP_SQRTY || o == QCB_OP_INVSQRTY; }
// no frame action
static bool is_frame_noop(uint32_t o) { return o == QCB_OP_I || o == QCB_OP_X || o == QCB_OP_Y || o == QCB_OP_Z; }

struct LOp {  // lowered op (0-based qubits)
  uint32_t kind;   // SegKind; SEG_END marks noise, SEG_H marks a relabel
  uint32_t opcode;
  uint32_t q1, q2;
  uint32_t bit;    // 0-based record row or BIT_NONE
  uint32_t reset;  // reset index (MRZ)
  int64_t site;    // noise site
  size_t src;      // index in the caller's op array
  uint32_t xa = 0, za = 0, xb = 0, zb = 0;  // planes, fixed when the op joins a segment
  std::vector<uint32_t> xin;  // ClassicalXOR: 0-based input record rows
};

static uint64_t fnv1a(const void* p, size_t n, uint64_t h = 1469598103934665603ull) {
  const uint8_t* b = (const uint8_t*)p;
  for (size_t i = 0; i < n; i++) { h ^= b[i]; h *= 1099511628211ull; }
  return h;
}

struct Emitter {
  std::vector<uint32_t>& out;
  std::vector<uint8_t>& swp;     // per slot: x currently lives in plane 2s+1
  std::vector<uint32_t>& slot;   // qubit -> slot
  uint32_t px(uint32_t q) const { uint32_t s = slot[q]; return 2 * s + (swp[s] ? 1 : 0); }
  uint32_t pz(uint32_t q) const { uint32_t s = slot[q]; return 2 * s + (swp[s] ? 0 : 1); }
  void pad4() { while (out.size() % 4) out.push_back(0); }
};

// Event probabilities of a noise site.  PauliNoise (src/pauli_frames.jl:157-174):
// X below px, Z below px+pz, Y below px+pz+py.  DepolarizationNoise(p) on k
// qubits (src/noise.jl:122-132): a uniform Pauli of the 4^k with probability p,
// so a non-identity one with p_eff = p (4^k-1)/4^k, uniform over those.
void fill_site_probabilities(Site& s, const qcb_op& op) {
  if (op.opcode == QCB_OP_PAULI_NOISE) {
    s.t0 = op.p[0];
    s.t1 = op.p[0] + op.p[2];
    s.t2 = op.p[0] + op.p[2] + op.p[1];
    s.peff = s.t2;
  } else {
    const double np = op.opcode == QCB_OP_DEPOL2 ? 15.0 : 3.0;
    s.peff = op.p[0] * np / (np + 1.0);
    s.t0 = s.t1 = s.t2 = s.peff;
  }
  if (s.peff > 1.0) s.peff = 1.0;
  s.dense = s.peff * NOISE_GROUP > NOISE_DENSE_LAMBDA ? 1u : 0u;
  if (s.peff < 1.0) {
    s.q0 = std::pow(1.0 - s.peff, (double)NOISE_GROUP);
    s.r = s.peff / (1.0 - s.peff);
  } else {
    s.q0 = 0.0;
    s.r = 0.0;
  }
}

// round(x * 2^bits), clamped to [0, 2^bits]; x * 2^bits is exact.
static uint64_t fixed_point(double x, uint32_t bits) {
  const double one = std::ldexp(1.0, (int)bits);
  const double f = std::floor(x * one + 0.5);
  if (!(f > 0.0)) return 0;
  return f >= one ? (uint64_t)1 << bits : (uint64_t)f;
}

// Fixed-point thresholds of a site's class (layout in qcb_internal.h).
static NoiseClass noise_class(const Site& s) {
  NoiseClass c{};
  c.dense = s.dense;
  c.np = s.kind == QCB_OP_DEPOL2 ? 15u : 3u;
  if (s.dense) {
    c.thr0 = fixed_point(s.t0, 32);
    c.thr1 = fixed_point(s.t1, 32);
    c.thr2 = fixed_point(std::min(s.t2, 1.0), 32);
  } else if (s.peff > 0.0) {
    // kind given an event: X with px / p_eff, Z with pz / p_eff, else Y
    c.thr0 = fixed_point(s.t0 / s.peff, NOISE_KIND_BITS);
    c.thr1 = fixed_point(s.t1 / s.peff, NOISE_KIND_BITS);
    c.thr2 = (uint64_t)1 << NOISE_KIND_BITS;
  }
  return c;
}

// Count thresholds of Binomial(NOISE_GROUP, p): entry k = round(P(K <= k) *
// 2^32), appended while below 2^32 (at most NOISE_CDF_MAX entries).  The pmf
// follows P(k+1) = P(k) (N-k)/(k+1) p/(1-p) from P(0) = (1-p)^N.
static void binomial_count_table(double p, std::vector<uint32_t>& out) {
  const double r = p / (1.0 - p);
  double pk = std::pow(1.0 - p, (double)NOISE_GROUP), cum = pk;
  for (uint32_t k = 0; k < NOISE_CDF_MAX; k++) {
    const uint64_t f = fixed_point(cum, 32);
    if (f >> 32) break;
    out.push_back((uint32_t)f);
    pk = pk * ((double)(NOISE_GROUP - k) * r) / (double)(k + 1);
    cum = cum + pk;
  }
}

int compile(const qcb_op* ops, size_t n_ops, Program& P) {
  std::memset(&P.info, 0, sizeof(P.info));
  P.info.n_ops = (uint32_t)n_ops;
  std::vector<LOp> low;
  low.reserve(n_ops + 16);
  P.site_of_op.assign(n_ops, -1);
  uint32_t nq = 0, nbits = 0, nresets = 0;
  uint64_t nsites = 0;
  for (size_t k = 0; k < n_ops; k++) {
    const qcb_op& op = ops[k];
    const uint32_t oc = op.opcode;
    const bool two = is2q(oc) || oc == QCB_OP_DEPOL2;
    if (!(is1q(oc) || is2q(oc) || isnoise(oc) || ismeas(oc) || oc == QCB_OP_NOP || oc == QCB_OP_XOR ||
          oc == QCB_OP_XOR_BITS))
      return fail(QCB_EUNSUPPORTED, "op " + std::to_string(k) + ": unknown opcode " + std::to_string(oc));
    if (oc == QCB_OP_NOP) continue;
    if (oc == QCB_OP_XOR_BITS)
      return fail(QCB_EARG, "op " + std::to_string(k) + ": ClassicalXOR input bits without their QCB_OP_XOR");
    if (oc == QCB_OP_XOR) {  // ClassicalXOR: the input bits follow in XOR_BITS ops
      const uint32_t n = op.q1;
      if (n < 1 || n > XOR_MAX_BITS)
        return fail(QCB_EUNSUPPORTED, "op " + std::to_string(k) + ": ClassicalXOR of " + std::to_string(n) +
                                          " bits (1.." + std::to_string(XOR_MAX_BITS) + " supported)");
      if (op.bit == 0) return fail(QCB_EBOUNDS, "op " + std::to_string(k) + ": ClassicalXOR store bit 0");
      const size_t npay = (n + 2) / 3;
      if (k + npay >= n_ops)
        return fail(QCB_EARG, "op " + std::to_string(k) + ": ClassicalXOR is missing its input bits");
      LOp x{SEG_XOR, oc, 0, 0, op.bit - 1, 0, -1, k};
      for (size_t j = 1; j <= npay; j++) {
        const qcb_op& pl = ops[k + j];
        if (pl.opcode != QCB_OP_XOR_BITS)
          return fail(QCB_EARG, "op " + std::to_string(k + j) + ": expected the ClassicalXOR's input bits");
        for (uint32_t b : {pl.q1, pl.q2, pl.bit})
          if (b && x.xin.size() < n) x.xin.push_back(b - 1);
      }
      if (x.xin.size() != n) return fail(QCB_EARG, "op " + std::to_string(k) + ": ClassicalXOR input bit 0");
      nbits = std::max(nbits, op.bit);
      for (uint32_t b : x.xin) nbits = std::max(nbits, b + 1);
      low.push_back(std::move(x));
      k += npay;
      continue;
    }
    if (op.q1 == 0 || (two && op.q2 == 0))
      return fail(QCB_EZEROQUBIT, "op " + std::to_string(k) + ": qubit indices start at 1 (NoZeroQubit)");
    if (two && op.q1 == op.q2)
      return fail(QCB_EARG, "op " + std::to_string(k) +
                                ": Failed to create a two qubit gate because the two qubits it acts on "
                                "have the same index. The qubit indices have to be different.");
    if (op.q1 > (1u << 30) || (two && op.q2 > (1u << 30)))
      return fail(QCB_EBOUNDS, "op " + std::to_string(k) + ": qubit index too large");
    nq = std::max(nq, op.q1);
    if (two) nq = std::max(nq, op.q2);
    const uint32_t q1 = op.q1 - 1, q2 = two ? op.q2 - 1 : 0;
    if (is1q(oc)) {
      P.info.n_updates++;
      if (is_frame_noop(oc)) continue;
      if (oc == QCB_OP_SQO) {  // by its bit map: nothing, x <-> z, z ^= x, or generic
        const uint32_t m = op.q2 & 15u;
        if (m == 9u) continue;  // xx, zz: identity on frames
        const uint32_t kind = m == 6u ? SEG_H : m == 11u ? SEG_S : SEG_G1;
        low.push_back({kind, QCB_OP_SQO | ((op.q2 & 63u) << 8), q1, 0, BIT_NONE, 0, -1, k});
        continue;
      }
      const uint32_t kind = is_relabel(oc) ? SEG_H : (oc == QCB_OP_S || oc == QCB_OP_SDAG || oc == QCB_OP_HXY) ? SEG_S : SEG_G1;
      low.push_back({kind, oc, q1, 0, BIT_NONE, 0, -1, k});
    } else if (is2q(oc)) {
      P.info.n_updates++;
      const uint32_t kind = (oc == QCB_OP_CNOT || oc == QCB_OP_ZCX) ? SEG_CNOT
                            : (oc == QCB_OP_CPHASE || oc == QCB_OP_ZCZ) ? SEG_CZ : SEG_G2;
      low.push_back({kind, oc, q1, q2, BIT_NONE, 0, -1, k});
    } else if (ismeas(oc)) {
      nbits = std::max(nbits, op.bit);
      const uint32_t bit = op.bit ? op.bit - 1 : BIT_NONE;
      P.info.n_updates++;
      if (oc == QCB_OP_MZ) {
        if (op.bit == 0) continue;  // src/pauli_frames.jl:86
        low.push_back({SEG_MZ, oc, q1, 0, bit, 0, -1, k});
      } else if (oc == QCB_OP_MX) {
        if (op.bit == 0) continue;  // src/pauli_frames.jl:75
        low.push_back({SEG_H, QCB_OP_H, q1, 0, BIT_NONE, 0, -1, k});
        low.push_back({SEG_MZ, QCB_OP_MZ, q1, 0, bit, 0, -1, k});
      } else if (oc == QCB_OP_MRZ) {
        low.push_back({SEG_MRZ, oc, q1, 0, bit, nresets++, -1, k});
      } else {  // MRX
        low.push_back({SEG_H, QCB_OP_H, q1, 0, BIT_NONE, 0, -1, k});
        low.push_back({SEG_MRZ, QCB_OP_MRZ, q1, 0, bit, nresets++, -1, k});
      }
    } else {  // noise
      for (int i = 0; i < 3; i++)
        if (!(op.p[i] >= 0.0) || !std::isfinite(op.p[i]))
          return fail(QCB_EARG, "op " + std::to_string(k) + ": noise probabilities must be finite and >= 0");
      P.site_of_op[k] = (int64_t)nsites;
      low.push_back({SEG_END, oc, q1, q2, BIT_NONE, 0, (int64_t)nsites, k});
      nsites++;
    }
  }
  if (nsites >= (1ull << 26)) return fail(QCB_EUNSUPPORTED, "too many noise sites (limit 2^26)");
  P.info.nqubits = nq;
  P.info.nbits = nbits;
  P.info.n_resets = nresets;
  P.info.n_noise_sites = (uint32_t)nsites;
  P.nq = nq;

  // slots: qubits in order of first use (relabels included)
  std::vector<uint32_t> qslot(nq + 1, BIT_NONE);
  P.slot_qubit.clear();
  auto touch = [&](uint32_t q) {
    if (qslot[q] == BIT_NONE) { qslot[q] = (uint32_t)P.slot_qubit.size(); P.slot_qubit.push_back(q); }
  };
  for (auto& o : low) {
    if (o.kind == SEG_XOR) continue;  // no qubits
    touch(o.q1);
    if (o.kind == SEG_CNOT || o.kind == SEG_CZ || o.kind == SEG_G2 || o.opcode == QCB_OP_DEPOL2) touch(o.q2);
  }
  P.nslots = (uint32_t)P.slot_qubit.size();
  std::vector<uint8_t> swp(P.nslots, 0);
  Emitter E{P.stream_slot, swp, qslot};
  P.stream_slot.clear();
  P.sites_slot.assign(nsites, Site{});
  P.site_arity.assign(nsites, 1);

  double pmax = 0;
  uint32_t nseg = 0, nflush = 0;
  if (2ull * P.nslots > 65536) return fail(QCB_EUNSUPPORTED, "at most 32768 distinct qubits per program");

  // Noise classes: sites of one opcode with equal probabilities share one
  // entry; sparse classes with equal p_eff share one count table.
  std::vector<NoiseClass> classes;
  std::vector<uint32_t> cdf;
  std::map<std::tuple<uint32_t, double, double, double, double>, uint32_t> class_of;
  std::map<double, std::pair<uint32_t, uint32_t>> table_of;
  auto class_id = [&](const Site& s) -> uint32_t {
    auto key = std::make_tuple(s.kind, s.t0, s.t1, s.t2, s.peff);
    auto it = class_of.find(key);
    if (it != class_of.end()) return it->second;
    NoiseClass c = noise_class(s);
    if (!c.dense && s.peff > 0.0) {
      auto t = table_of.find(s.peff);
      if (t == table_of.end()) {
        while (cdf.size() % 4) cdf.push_back(0xFFFFFFFFu);  // tables start on 16 bytes (read 4 at a time)
        const uint32_t off = (uint32_t)cdf.size();
        binomial_count_table(s.peff, cdf);
        t = table_of.emplace(s.peff, std::make_pair(off, (uint32_t)cdf.size() - off)).first;
      }
      c.cdf_off = t->second.first;
      c.cdf_len = t->second.second;
    }
    classes.push_back(c);
    return class_of[key] = (uint32_t)(classes.size() - 1);
  };

  // Records before windowing: fixed-size entries of one kind.
  struct Rec { uint32_t kind, entry_words; std::vector<uint32_t> w; };
  std::vector<Rec> recs;
  auto pk = [](uint32_t a, uint32_t b) { return a | (b << 16); };
  auto emit_seg = [&](uint32_t kind, std::vector<LOp>& seg) {
    if (seg.empty()) return;
    Rec r{kind, 2, {}};
    switch (kind) {
      case SEG_CNOT:
      case SEG_CZ:  // (x_a | z_a << 16, x_b | z_b << 16)
        for (auto& o : seg) { r.w.push_back(pk(o.xa, o.za)); r.w.push_back(pk(o.xb, o.zb)); }
        break;
      case SEG_S:
      case SEG_G1:  // (x | z << 16, opcode)
        for (auto& o : seg) { r.w.push_back(pk(o.xa, o.za)); r.w.push_back(o.opcode); }
        break;
      case SEG_G2:  // (x_a | z_a << 16, x_b | z_b << 16, opcode, 0)
        r.entry_words = 4;
        for (auto& o : seg) { r.w.push_back(pk(o.xa, o.za)); r.w.push_back(pk(o.xb, o.zb)); r.w.push_back(o.opcode); r.w.push_back(0); }
        break;
      case SEG_MZ:  // (x, bit)
        for (auto& o : seg) { r.w.push_back(o.xa); r.w.push_back(o.bit); }
        break;
      case SEG_XOR:  // (store, n, b_0 .. b_{n-1}, 0 ...)
        r.entry_words = 32;
        for (auto& o : seg) {
          r.w.push_back(o.bit);
          r.w.push_back((uint32_t)o.xin.size());
          for (uint32_t i = 0; i < 30; i++) r.w.push_back(i < o.xin.size() ? o.xin[i] : 0u);
        }
        break;
      case SEG_MRZ: {  // groups of 4 entries (x | z << 16, bit, reset | PAD, 0); entry i of a group
                       // holds reset 4*block + i, so one Philox block serves the group
        r.entry_words = 16;
        std::sort(seg.begin(), seg.end(), [](const LOp& a, const LOp& b) { return a.reset < b.reset; });
        size_t i = 0;
        while (i < seg.size()) {
          const uint32_t blk = seg[i].reset >> 2;
          const LOp* ent[4] = {nullptr, nullptr, nullptr, nullptr};
          while (i < seg.size() && (seg[i].reset >> 2) == blk) { ent[seg[i].reset & 3] = &seg[i]; i++; }
          for (int k = 0; k < 4; k++) {
            const LOp* o = ent[k];
            if (o) { r.w.push_back(pk(o->xa, o->za)); r.w.push_back(o->bit); r.w.push_back(o->reset); r.w.push_back(0); }
            else { r.w.push_back(0); r.w.push_back(BIT_NONE); r.w.push_back(MRZ_PAD); r.w.push_back(0); }
          }
        }
        break;
      }
      default: break;
    }
    recs.push_back(std::move(r));
    nseg++;
  };
  // FLUSH: one entry per site (site, kind | class << 8, x_a | z_a << 16, x_b | z_b << 16).
  auto emit_sites = [&](std::vector<uint32_t>& st) {
    if (st.empty()) return;
    std::sort(st.begin(), st.end());
    Rec r{SEG_FLUSH, 4, {}};
    for (uint32_t si : st) {
      const Site& s = P.sites_slot[si];
      r.w.push_back(si);
      r.w.push_back(s.kind | (class_id(s) << 8));
      r.w.push_back(pk(s.xa, s.za));
      r.w.push_back(pk(s.xb, s.zb));
    }
    recs.push_back(std::move(r));
    nflush++;
    st.clear();
  };

  // Scheduling, in program order.  The open segment collects ops of one kind
  // on pairwise-disjoint qubits.  A noise op goes to the open segment's
  // pre-flush (applied before the segment) when the segment does not touch its
  // qubits -- every earlier op on them is in an emitted segment -- and
  // otherwise to the post-flush, which is applied before the next segment.  An
  // op that touches a qubit with post-flush noise, overlaps the segment, writes
  // a record bit the segment writes, or has another kind closes the segment.
  // Flips commute with ops on other qubits, so the result equals op-by-op
  // execution, and a circuit written in layers (noise after each gate,
  // measurement flips before each reset) gets one flush per layer.
  std::vector<LOp> cur;
  uint32_t cur_kind = SEG_END;
  std::unordered_set<uint32_t> cur_q, post_q, cur_bits, cur_reads;
  std::vector<uint32_t> pre, post;
  auto close_seg = [&]() {
    emit_sites(pre);
    emit_seg(cur_kind, cur);
    cur.clear();
    cur_q.clear();
    cur_bits.clear();
    cur_reads.clear();
    cur_kind = SEG_END;
    pre.swap(post);
    post_q.clear();
  };
  for (auto& o : low) {
    if (o.kind == SEG_END) {  // noise: record the site with the current planes
      const qcb_op& op = ops[o.src];
      Site& s = P.sites_slot[(size_t)o.site];
      s.kind = op.opcode;
      s.xa = E.px(o.q1); s.za = E.pz(o.q1);
      bool touches = cur_q.count(o.q1) > 0;
      if (op.opcode == QCB_OP_DEPOL2) {
        s.xb = E.px(o.q2); s.zb = E.pz(o.q2);
        touches = touches || cur_q.count(o.q2) > 0;
        P.site_arity[(size_t)o.site] = 2;
      }
      fill_site_probabilities(s, op);
      pmax = std::max(pmax, s.peff);
      if (touches) {
        post.push_back((uint32_t)o.site);
        post_q.insert(o.q1);
        if (op.opcode == QCB_OP_DEPOL2) post_q.insert(o.q2);
      } else {
        pre.push_back((uint32_t)o.site);
      }
      continue;
    }
    if (o.kind == SEG_H) {  // relabel x <-> z of this qubit, no run-time work
      swp[qslot[o.q1]] ^= 1;
      continue;
    }
    if (o.kind == SEG_XOR) {
      // record rows only: a segment of XORs may not read a row it stores, nor
      // store a row it reads or stores already
      bool dep = cur_bits.count(o.bit) || cur_reads.count(o.bit);
      for (uint32_t b : o.xin) dep = dep || cur_bits.count(b);
      if (!cur.empty() && (dep || cur_kind != SEG_XOR)) close_seg();
      cur_kind = SEG_XOR;
      cur.push_back(o);
      cur_bits.insert(o.bit);
      for (uint32_t b : o.xin) cur_reads.insert(b);
      continue;
    }
    const bool two = o.kind == SEG_CNOT || o.kind == SEG_CZ || o.kind == SEG_G2;
    const bool hit = post_q.count(o.q1) || (two && post_q.count(o.q2));
    const bool overlap = cur_q.count(o.q1) || (two && cur_q.count(o.q2));
    const bool same_bit = o.bit != BIT_NONE && cur_bits.count(o.bit);
    if (!cur.empty() && (hit || overlap || same_bit || o.kind != cur_kind)) close_seg();
    cur_kind = o.kind;
    LOp c = o;  // planes current at this op
    c.xa = E.px(o.q1); c.za = E.pz(o.q1);
    if (two) { c.xb = E.px(o.q2); c.zb = E.pz(o.q2); }
    cur.push_back(c);
    cur_q.insert(o.q1);
    if (two) cur_q.insert(o.q2);
    if (o.bit != BIT_NONE) cur_bits.insert(o.bit);
  }
  close_seg();
  emit_sites(pre);

  // Windowing: the kernel stages the stream into shared memory one window
  // (8 or 16 KB, below) at a time, so no record may straddle a window.  A record
  // too long for the space left is split into parts (entries of one segment
  // or flush are independent; every part but the last is marked so that no
  // barrier follows it); a window ends with a WIN record, the stream with END.
  // Window size: 16 KB for a program with a record longer than an 8 KB
  // window and a frame of 512..1536 slots (its tiles are narrow, so 8 KB
  // more staging costs a few columns, while every split record costs a walk
  // step: d=25 15.2 -> 13.7 ms; up to 1536 slots a 16-column shared-memory
  // tile still fits next to 16 KB windows), 8 KB otherwise (d=11 keeps its
  // 106-column tiles).  The WIN record carries the size.
  size_t longest = 0;
  for (auto& r : recs) longest = std::max(longest, 4 + ((r.w.size() + 3) & ~(size_t)3));
  const bool tall = longest > PROG_WINDOW_WORDS - 4 && P.nslots >= 512 && P.nslots <= 1536;
  const uint32_t W = tall ? PROG_WINDOW_WORDS_TALL : PROG_WINDOW_WORDS;
  P.win_words = W;
  auto& out = P.stream_slot;
  out.clear();
  auto room = [&]() { return W - (uint32_t)(out.size() % W) - 4; };
  auto next_window = [&]() {
    out.push_back((SEG_WIN << 24) | W); out.push_back(0); out.push_back(0); out.push_back(0);
    while (out.size() % W) out.push_back(0);
  };
  P.pre_ent.clear();
  P.pre_capoff.assign(1, 0);
  P.pre_nparts = 0;
  for (auto& r : recs) {
    const uint32_t n = (uint32_t)(r.w.size() / r.entry_words);
    // A record that fits one window is not split: it starts the next window
    // when the rest of this one is too small.  Every part of a split record
    // is one more step of the walk, with a CTA barrier before it and, for a
    // flush, one more dependent sampling chain; padding costs only words.
    const size_t whole = 4 + ((r.w.size() + 3) & ~(size_t)3);
    if (whole <= W - 4 && whole > room()) next_window();
    uint32_t done = 0;
    while (done < n) {
      if (room() < 4 + ((r.entry_words + 3) & ~3u)) next_window();
      const uint32_t fit = (room() - 4) / r.entry_words;
      // room() - 4 is a multiple of 4 words, so the padded part fits too
      const uint32_t take = std::min(n - done, fit);
      const bool last = done + take == n;
      uint32_t aux0 = last ? 0u : FLAG_NO_BARRIER, aux1 = 0, aux2 = 0;
      if (r.kind == SEG_FLUSH) {
        // flush part j (header word 2); its sparse sites go to the
        // pre-sampler's entry table, dense ones are drawn in the walk (header
        // word 3 bit 0).  Bucket capacity per group: the expected event count
        // Lambda plus 8 standard deviations and a margin (a bucket that
        // overflows is drawn in the walk instead, so this bounds memory only).
        const uint32_t j = P.pre_nparts++;
        double lam = 0;
        for (uint32_t t = 0; t < take; t++) {
          const uint32_t* en = &r.w[(size_t)(done + t) * 4];
          const NoiseClass& c = classes[en[1] >> 8];
          if (c.dense) { aux0 |= FLAG_DENSE_SITES; continue; }
          if (!c.cdf_len) continue;
          P.pre_ent.push_back(make_uint4(en[0], en[1], j, t));
          lam += P.sites_slot[en[0]].peff * NOISE_GROUP;
        }
        const uint32_t cap = lam > 0 ? ((uint32_t)std::ceil(lam + 8.0 * std::sqrt(lam) + 32.0) + 3u) & ~3u : 0u;
        if (cap >= (1u << 24)) return fail(QCB_EUNSUPPORTED, "noise pre-sampling: a flush part expects too many events");
        aux0 |= cap << 8;                 // header word 1: flags | bucket capacity << 8
        aux1 = j;                         // header word 2: the part
        aux2 = P.pre_capoff.back();       // header word 3: the bucket's offset in a group's events
        P.pre_capoff.push_back(P.pre_capoff.back() + cap);
      }
      out.push_back((r.kind << 24) | take);
      out.push_back(aux0); out.push_back(aux1); out.push_back(aux2);
      out.insert(out.end(), r.w.begin() + (size_t)done * r.entry_words, r.w.begin() + (size_t)(done + take) * r.entry_words);
      while (out.size() % 4) out.push_back(0);
      done += take;
    }
  }
  out.push_back(SEG_END << 24); out.push_back(0); out.push_back(0); out.push_back(0);
  while (out.size() % W) out.push_back(0);
  P.classes = classes;
  while (cdf.size() % 4) cdf.push_back(0xFFFFFFFFu);  // the last 4-word read stays inside
  P.cdf = cdf;
  P.info.n_segments = nseg;
  P.info.n_flushes = nflush;
  P.slot_swap.assign(swp.begin(), swp.end());
  P.pmax = pmax;
  P.hash = fnv1a(ops, n_ops * sizeof(qcb_op));
  return QCB_OK;
}

int upload(Program& P) {
  // device copies
  auto up = [&](auto** dptr, const auto& vec) -> cudaError_t {
    size_t bytes = vec.size() * sizeof(vec[0]);
    cudaError_t e = cudaMalloc((void**)dptr, bytes ? bytes : 16);
    if (e != cudaSuccess) return e;
    if (bytes) e = cudaMemcpy(*dptr, vec.data(), bytes, cudaMemcpyHostToDevice);
    return e;
  };
  cudaError_t e = up(&P.d_stream_slot, P.stream_slot);
  if (e == cudaSuccess) e = up(&P.d_classes, P.classes);
  if (e == cudaSuccess) e = up(&P.d_cdf, P.cdf);
  if (e == cudaSuccess) e = up(&P.d_slot_qubit, P.slot_qubit);
  std::vector<uint32_t> qs(P.nq + 1, BIT_NONE);
  for (uint32_t s = 0; s < P.nslots; s++) qs[P.slot_qubit[s]] = s;
  P.qubit_slot_len = (uint32_t)qs.size();
  if (e == cudaSuccess) e = up(&P.d_qubit_slot, qs);
  std::vector<uint32_t> sw(P.slot_swap.begin(), P.slot_swap.end());
  if (e == cudaSuccess) e = up(&P.d_slot_swap, sw);
  if (e == cudaSuccess) e = up(&P.d_pre_ent, P.pre_ent);
  if (e == cudaSuccess) e = up(&P.d_pre_capoff, P.pre_capoff);
  if (e != cudaSuccess) return cuda_fail(e, "qcb_program_compile upload");
  return QCB_OK;
}

void release(Program& P) {
  cudaFree(P.d_stream_slot);
  cudaFree(P.d_classes);
  cudaFree(P.d_cdf);
  cudaFree(P.d_slot_qubit);
  cudaFree(P.d_qubit_slot);
  cudaFree(P.d_slot_swap);
  cudaFree(P.d_pre_ent);
  cudaFree(P.d_pre_capoff);
  P.d_pre_ent = nullptr;
  P.d_pre_capoff = nullptr;
  P.d_stream_slot = nullptr;
  P.d_classes = nullptr;
  P.d_cdf = nullptr;
  P.d_slot_qubit = P.d_qubit_slot = P.d_slot_swap = nullptr;
}

}  // namespace qcb

using namespace qcb;

extern "C" {

int qcb_program_compile(const qcb_op* ops, size_t n_ops, qcb_program** out) {
  if (!out) return fail(QCB_EARG, "qcb_program_compile: null out");
  *out = nullptr;
  if (n_ops && !ops) return fail(QCB_EARG, "qcb_program_compile: null ops");
  qcb_program* p = new qcb_program();
  int st = compile(ops, n_ops, *p);
  if (st == QCB_OK) st = upload(*p);
  if (st != QCB_OK) { release(*p); delete p; return st; }
  *out = p;
  return QCB_OK;
}

int qcb_debug_program_dump(const qcb_op* ops, size_t n_ops, uint32_t* stream, size_t stream_cap,
                           size_t* stream_len, uint8_t* sites, size_t sites_cap, size_t* n_sites,
                           uint32_t* slot_qubit, uint32_t* slot_swap, size_t slots_cap, size_t* n_slots,
                           qcb_program_info* info) {
  Program P;
  int st = compile(ops, n_ops, P);
  if (st != QCB_OK) return st;
  if (stream_len) *stream_len = P.stream_slot.size();
  if (n_sites) *n_sites = P.sites_slot.size();
  if (n_slots) *n_slots = P.nslots;
  if (info) *info = P.info;
  if (stream && stream_cap >= P.stream_slot.size())
    std::memcpy(stream, P.stream_slot.data(), P.stream_slot.size() * 4);
  if (sites && sites_cap >= P.sites_slot.size() * sizeof(Site))
    std::memcpy(sites, P.sites_slot.data(), P.sites_slot.size() * sizeof(Site));
  if (slots_cap >= P.nslots) {
    for (uint32_t s = 0; s < P.nslots; s++) {
      if (slot_qubit) slot_qubit[s] = P.slot_qubit[s];
      if (slot_swap) slot_swap[s] = P.slot_swap[s];
    }
  }
  return QCB_OK;
}

int qcb_program_info_get(const qcb_program* prog, qcb_program_info* info) {
  if (!prog || !info) return fail(QCB_EARG, "null argument");
  *info = prog->info;
  return QCB_OK;
}

int qcb_program_device_bytes(const qcb_program* prog, uint64_t* bytes) {
  if (!prog || !bytes) return fail(QCB_EARG, "null argument");
  *bytes = prog->stream_slot.size() * sizeof(uint32_t) + prog->classes.size() * sizeof(NoiseClass) +
           prog->cdf.size() * sizeof(uint32_t);
  return QCB_OK;
}

int qcb_program_destroy(qcb_program* prog) {
  if (!prog) return QCB_OK;
  release(*prog);
  delete prog;
  return QCB_OK;
}

}  // extern "C"
