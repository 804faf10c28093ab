// program.cu -- circuit -> device program compiler.
//
// Replaces the per-op dispatch of pftrajectories(frame, circuit)
// (src/pauli_frames.jl:234-239) and compactify_circuit (src/sumtypes.jl:190-237).
// Ops are validated like the Julia constructors (NoZeroQubit, q1 == q2),
// sMX / sMRX are lowered to sHadamard + sMZ / sMRZ (src/pauli_frames.jl:74-83),
// and the remaining ops are grouped into segments: runs of one gate kind on
// pairwise-disjoint qubits, which the walker kernel executes with independent
// loads in flight.  Noise ops do not break segments; they are collected into
// a pending set and applied at a FLUSH record placed before the first later
// op that touches one of their qubits.  Moving a Pauli flip past gates that act
// on other qubits is exact, so the result equals op-by-op execution.
#include <cmath>
#include <cstring>
#include <unordered_set>

#include "qcb_internal.h"

namespace qcb {

static bool is1q(uint32_t o) { return o >= QCB_OP_I && o <= QCB_OP_CZYX; }
static bool is2q(uint32_t o) { return o >= QCB_OP_CNOT && o <= QCB_OP_YCZ; }
static bool isnoise(uint32_t o) { return o >= QCB_OP_PAULI_NOISE && o <= QCB_OP_DEPOL2; }
static bool ismeas(uint32_t o) { return o >= QCB_OP_MZ && o <= QCB_OP_MRX; }

struct LOp {  // lowered op (0-based qubits)
  uint32_t kind;   // SegKind for gates/measurements; 0 for noise
  uint32_t opcode;
  uint32_t q1, q2;
  uint32_t bit;    // 0-based record row or BIT_NONE
  uint32_t reset;  // reset index (MRZ)
  int64_t site;    // noise site (noise ops)
};

static uint64_t fnv1a(const void* p, size_t n, uint64_t h = 1469598103934665603ull) {
  const uint8_t* b = (const uint8_t*)p;
  for (size_t i = 0; i < n; i++) { h ^= b[i]; h *= 1099511628211ull; }
  return h;
}

static void emit_segment(std::vector<uint32_t>& out, uint32_t kind, const std::vector<LOp>& ops,
                         const std::vector<uint32_t>& map, uint32_t scratch) {
  auto M = [&](uint32_t q) { return map.empty() ? q : map[q]; };
  uint32_t cnt = (uint32_t)ops.size();
  out.push_back((kind << 24) | cnt);
  out.push_back(0); out.push_back(0); out.push_back(0);
  switch (kind) {
    case SEG_CNOT: case SEG_CZ: {
      for (auto& o : ops) { out.push_back(M(o.q1)); out.push_back(M(o.q2)); }
      // pad with gates on the scratch slot to a multiple of 4 gates
      for (uint32_t i = cnt; i % 4; i++) { out.push_back(scratch); out.push_back(scratch); }
      break;
    }
    case SEG_H: case SEG_S: {
      for (auto& o : ops) out.push_back(M(o.q1));
      for (uint32_t i = cnt; i % 4; i++) out.push_back(scratch);
      break;
    }
    case SEG_G1: {
      for (auto& o : ops) { out.push_back(o.opcode); out.push_back(M(o.q1)); }
      for (uint32_t i = cnt; i % 2; i++) { out.push_back(QCB_OP_I); out.push_back(scratch); }
      break;
    }
    case SEG_G2: {
      for (auto& o : ops) {
        out.push_back(o.opcode); out.push_back(M(o.q1)); out.push_back(M(o.q2)); out.push_back(0);
      }
      break;
    }
    case SEG_MZ: {
      for (auto& o : ops) { out.push_back(M(o.q1)); out.push_back(o.bit); }
      for (uint32_t i = cnt; i % 2; i++) { out.push_back(scratch); out.push_back(BIT_NONE); }
      break;
    }
    case SEG_MRZ: {
      for (auto& o : ops) {
        out.push_back(M(o.q1)); out.push_back(o.bit); out.push_back(o.reset); out.push_back(0);
      }
      break;
    }
    default: break;
  }
}

static void emit_flush(std::vector<uint32_t>& out, uint32_t sb, uint32_t se) {
  out.push_back((SEG_FLUSH << 24));
  out.push_back(sb); out.push_back(se); out.push_back(0);
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
    uint32_t oc = op.opcode;
    bool two = is2q(oc) || oc == QCB_OP_DEPOL2;
    if (!(is1q(oc) || is2q(oc) || isnoise(oc) || ismeas(oc) || oc == QCB_OP_NOP))
      return fail(QCB_EUNSUPPORTED, "op " + std::to_string(k) + ": unknown opcode " + std::to_string(oc));
    if (oc == QCB_OP_NOP) continue;
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
    uint32_t q1 = op.q1 - 1, q2 = two ? op.q2 - 1 : 0;
    if (is1q(oc)) {
      uint32_t kind = oc == QCB_OP_H ? SEG_H : oc == QCB_OP_S ? SEG_S : SEG_G1;
      low.push_back({kind, oc, q1, 0, BIT_NONE, 0, -1});
      P.info.n_updates++;
    } else if (is2q(oc)) {
      uint32_t kind = oc == QCB_OP_CNOT ? SEG_CNOT : oc == QCB_OP_CPHASE ? SEG_CZ : SEG_G2;
      low.push_back({kind, oc, q1, q2, BIT_NONE, 0, -1});
      P.info.n_updates++;
    } else if (ismeas(oc)) {
      nbits = std::max(nbits, op.bit);
      uint32_t bit = op.bit ? op.bit - 1 : BIT_NONE;
      P.info.n_updates++;
      if (oc == QCB_OP_MZ) {
        if (op.bit == 0) continue;  // src/pauli_frames.jl:86
        low.push_back({SEG_MZ, oc, q1, 0, bit, 0, -1});
      } else if (oc == QCB_OP_MX) {
        if (op.bit == 0) continue;  // src/pauli_frames.jl:75
        low.push_back({SEG_H, QCB_OP_H, q1, 0, BIT_NONE, 0, -1});
        low.push_back({SEG_MZ, QCB_OP_MZ, q1, 0, bit, 0, -1});
      } else if (oc == QCB_OP_MRZ) {
        low.push_back({SEG_MRZ, oc, q1, 0, bit, nresets++, -1});
      } else {  // MRX
        low.push_back({SEG_H, QCB_OP_H, q1, 0, BIT_NONE, 0, -1});
        low.push_back({SEG_MRZ, QCB_OP_MRZ, q1, 0, bit, nresets++, -1});
      }
    } else {  // noise
      for (int i = 0; i < 3; i++)
        if (!(op.p[i] >= 0.0) || !std::isfinite(op.p[i]))
          return fail(QCB_EARG, "op " + std::to_string(k) + ": noise probabilities must be finite and >= 0");
      P.site_of_op[k] = (int64_t)nsites;
      low.push_back({0, oc, q1, q2, BIT_NONE, 0, (int64_t)nsites});
      nsites++;
    }
  }
  if (nsites >= (1ull << 26)) return fail(QCB_EUNSUPPORTED, "too many noise sites (limit 2^26)");
  P.info.nqubits = nq;
  P.info.nbits = nbits;
  P.info.n_resets = nresets;
  P.info.n_noise_sites = (uint32_t)nsites;
  P.nq = nq;

  // slot assignment: qubits in order of first use
  std::vector<uint32_t> qslot(nq + 1, BIT_NONE);
  P.slot_qubit.clear();
  auto touch = [&](uint32_t q) {
    if (qslot[q] == BIT_NONE) { qslot[q] = (uint32_t)P.slot_qubit.size(); P.slot_qubit.push_back(q); }
  };
  for (auto& o : low) {
    touch(o.q1);
    if (o.kind == SEG_CNOT || o.kind == SEG_CZ || o.kind == SEG_G2 || o.opcode == QCB_OP_DEPOL2) touch(o.q2);
  }
  P.nslots = (uint32_t)P.slot_qubit.size();
  std::vector<uint32_t> slotmap(qslot.begin(), qslot.end());

  // site table (operands in slot space)
  P.sites_slot.clear(); P.site_arity.clear();
  double pmax = 0;
  for (size_t k = 0; k < n_ops; k++) {
    if (P.site_of_op[k] < 0) continue;
    const qcb_op& op = ops[k];
    Site s{};
    s.kind = op.opcode;
    s.a = slotmap[op.q1 - 1];
    s.b = op.opcode == QCB_OP_DEPOL2 ? slotmap[op.q2 - 1] : 0;
    double pe;
    if (op.opcode == QCB_OP_PAULI_NOISE) {
      s.t0 = op.p[0]; s.t1 = op.p[0] + op.p[2]; s.t2 = op.p[0] + op.p[2] + op.p[1];
      pe = s.t2;
      P.site_arity.push_back(1);
    } else {
      double np = op.opcode == QCB_OP_DEPOL2 ? 15.0 : 3.0;
      s.t0 = op.p[0] * np / (np + 1.0);
      pe = s.t0;
      P.site_arity.push_back(op.opcode == QCB_OP_DEPOL2 ? 2 : 1);
    }
    if (pe > 1.0) pe = 1.0;
    pmax = std::max(pmax, pe);
    P.sites_slot.push_back(s);
  }
  P.pmax = pmax;
  P.inv_log1m = (pmax > 0 && pmax < 1.0) ? 1.0 / std::log1p(-pmax) : 0.0;

  // segmentation
  P.stream_slot.clear();
  std::vector<LOp> cur;
  uint32_t cur_kind = SEG_END;
  std::unordered_set<uint32_t> cur_q, pend_q;
  uint32_t pend_begin = 0, pend_end = 0;
  uint32_t nseg = 0, nflush = 0;
  auto close_seg = [&]() {
    if (cur.empty()) return;
    emit_segment(P.stream_slot, cur_kind, cur, slotmap, P.nslots);
    nseg++;
    cur.clear(); cur_q.clear(); cur_kind = SEG_END;
  };
  auto flush = [&]() {
    if (pend_end > pend_begin) {
      emit_flush(P.stream_slot, pend_begin, pend_end);
      nflush++;
    }
    pend_begin = pend_end;
    pend_q.clear();
  };
  for (auto& o : low) {
    bool two = o.kind == SEG_CNOT || o.kind == SEG_CZ || o.kind == SEG_G2;
    if (o.kind == 0) {  // noise
      pend_q.insert(o.q1);
      if (o.opcode == QCB_OP_DEPOL2) pend_q.insert(o.q2);
      pend_end = (uint32_t)o.site + 1;
      continue;
    }
    bool hit = pend_q.count(o.q1) || (two && pend_q.count(o.q2));
    if (hit) { close_seg(); flush(); }
    bool overlap = cur_q.count(o.q1) || (two && cur_q.count(o.q2));
    if (o.kind != cur_kind || overlap || cur.size() >= (1u << 20)) close_seg();
    cur_kind = o.kind;
    cur.push_back(o);
    cur_q.insert(o.q1);
    if (two) cur_q.insert(o.q2);
  }
  close_seg();
  flush();
  P.stream_slot.push_back(SEG_END << 24); P.stream_slot.push_back(0);
  P.stream_slot.push_back(0); P.stream_slot.push_back(0);
  P.info.n_segments = nseg;
  P.info.n_flushes = nflush;
  P.hash = fnv1a(ops, n_ops * sizeof(qcb_op));

  // device copies
  auto up = [&](auto** dptr, const auto& vec) -> cudaError_t {
    size_t bytes = vec.size() * sizeof(vec[0]);
    cudaError_t e = cudaMalloc((void**)dptr, bytes ? bytes : 16);
    if (e != cudaSuccess) return e;
    if (bytes) e = cudaMemcpy(*dptr, vec.data(), bytes, cudaMemcpyHostToDevice);
    return e;
  };
  cudaError_t e = up(&P.d_stream_slot, P.stream_slot);
  if (e == cudaSuccess) e = up(&P.d_sites_slot, P.sites_slot);
  if (e == cudaSuccess) e = up(&P.d_slot_qubit, P.slot_qubit);
  std::vector<uint32_t> qs(qslot.begin(), qslot.end());
  P.qubit_slot_len = (uint32_t)qs.size();
  if (e == cudaSuccess) e = up(&P.d_qubit_slot, qs);
  if (e != cudaSuccess) return cuda_fail(e, "qcb_program_compile upload");
  return QCB_OK;
}

void release(Program& P) {
  cudaFree(P.d_stream_slot);
  cudaFree(P.d_sites_slot);
  cudaFree(P.d_slot_qubit); cudaFree(P.d_qubit_slot);
  P.d_stream_slot = nullptr;
  P.d_sites_slot = nullptr;
  P.d_slot_qubit = P.d_qubit_slot = nullptr;
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
  if (st != QCB_OK) { release(*p); delete p; return st; }
  *out = p;
  return QCB_OK;
}

int qcb_program_info_get(const qcb_program* prog, qcb_program_info* info) {
  if (!prog || !info) return fail(QCB_EARG, "null argument");
  *info = prog->info;
  return QCB_OK;
}

int qcb_program_destroy(qcb_program* prog) {
  if (!prog) return QCB_OK;
  release(*prog);
  delete prog;
  return QCB_OK;
}

}  // extern "C"
